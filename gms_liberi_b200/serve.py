"""Continuous-batching Fock-build server over the engine's C ABI.

A *session* is one molecule's SCF run: `niter` Fock builds, the density
updated between builds.  Sessions arrive over time; the server

  * admits a waiting session (FIFO) as soon as a slot is free and its device
    footprint fits the HBM budget.  The footprint is exact and known before
    any allocation: the library's host-only dry run (`liberi_c_setup_bytes`)
    plus the session's own packed D and F;
  * keeps the session's shell pairs, Schwarz table, plans, D and F resident
    for all of its builds (one engine handle per session) and releases them
    when its last build completes;
  * launches every ready build immediately on the session's own CUDA stream,
    so builds of different sessions overlap on the device (continuous
    batching: new sessions join while others are in flight);
  * records, per build, the latency from its request (session arrival for the
    first build, completion of the previous build afterwards) to the moment
    its F is complete;
  * cancels sessions on request (`cancel(sid)` from any thread, or a
    session's scripted `cancel_at` time): a queued session leaves the queue
    without being set up; an admitted one finishes the build it has on the
    GPU (device work is not aborted), launches no more and releases its
    memory.

The scheduling logic is independent of the engine (`Engine` below), so it is
tested on the CPU with a fake engine; `LiberiEngine` drives the CUDA library.
Session setup (host planning, device upload) runs on a small pool of worker
threads (`setup_workers`), so the dispatch loop keeps launching builds and
sessions admitted together are set up side by side.
"""
import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Session:
    sid: int
    basis: dict
    niter: int
    seed: int
    arrival: float
    D0: object = None           # initial packed density (host), supplied with the request
    nbytes: int = 0
    state: object = None
    it: int = 0                 # builds completed
    t_request: float = 0.0      # request time of the build in flight / next build
    token: object = None        # engine token of the build in flight
    admitted_at: float = -1.0
    ready_at: float = -1.0      # setup finished
    waited: bool = False        # found the slots or the HBM budget full on arrival
    waited_bytes: bool = False  # held back by the HBM budget while a slot was free
    cancel_at: float = -1.0     # scripted cancellation time (s from the start), < 0: none
    cancelled: bool = False
    latencies: list = field(default_factory=list)
    results: list = field(default_factory=list)


class Engine:
    """What the server needs from an engine (the CUDA one is LiberiEngine)."""

    def bytes_needed(self, basis):
        raise NotImplementedError

    def open(self, session):          # allocate and set up; returns state
        raise NotImplementedError

    def launch(self, session):        # enqueue build `session.it`; returns a token
        raise NotImplementedError

    def done(self, token):            # has that build completed?
        raise NotImplementedError

    def result(self, session):        # F of the last completed build (tests)
        raise NotImplementedError

    def advance(self, session):       # density update for the next build
        raise NotImplementedError

    def close(self, session):
        raise NotImplementedError


class FockServer:
    def __init__(self, engine, hbm_budget, max_slots=64, capture=False, poll_s=2e-4, setup_workers=4):
        self.engine = engine
        self.setup_workers = max(1, int(setup_workers))
        self.budget = int(hbm_budget)
        self.max_slots = int(max_slots)
        self.capture = capture
        self.poll_s = poll_s
        self._cancel = set()
        self._cancel_lock = threading.Lock()

    def cancel(self, sid):
        """Request cancellation of session `sid` (thread-safe; takes effect at
        the loop's next pass)."""
        with self._cancel_lock:
            self._cancel.add(int(sid))

    def _cancelled(self, s, t):
        if s.cancel_at >= 0 and t >= s.cancel_at:
            return True
        with self._cancel_lock:
            return s.sid in self._cancel

    def run(self, arrivals, clock=time.perf_counter):
        """Serve `arrivals` (Sessions with arrival times in seconds from the
        start, ascending); returns the report and the finished sessions."""
        t0 = clock()
        now = lambda: clock() - t0
        pending = collections.deque(sorted(arrivals, key=lambda s: s.arrival))
        for s in pending:
            s.nbytes = int(self.engine.bytes_needed(s.basis))
            if s.nbytes > self.budget:
                raise ValueError("session %d needs %d bytes, above the HBM budget %d" % (s.sid, s.nbytes, self.budget))
        waiting = collections.deque()
        active, finished, cancelled = [], [], []
        reserved = peak_reserved = 0
        peak_active = 0
        in_setup = 0                       # admitted, handed to the worker, not back yet
        setup_q = collections.deque()      # loop -> worker
        setup_done = collections.deque()   # worker -> loop
        lock = threading.Condition()
        stop = [False]
        errors = []

        def worker():
            while True:
                with lock:
                    while not setup_q and not stop[0]:
                        lock.wait()
                    if not setup_q:
                        return
                    s = setup_q.popleft()
                try:
                    s.state = self.engine.open(s)
                except Exception as e:  # re-raised by the loop
                    errors.append(e)
                s.ready_at = now()
                with lock:
                    setup_done.append(s)

        ths = [threading.Thread(target=worker, daemon=True) for _ in range(self.setup_workers)]
        for th in ths:
            th.start()
        try:
            while pending or waiting or active or in_setup:
                if errors:
                    raise errors[0]
                t = now()
                while pending and pending[0].arrival <= t:
                    waiting.append(pending.popleft())
                # cancelled before admission: leave the queue, never set up
                for q in (pending, waiting):
                    for s in [x for x in q if self._cancelled(x, t)]:
                        q.remove(s)
                        s.cancelled = True
                        cancelled.append(s)
                # admission: FIFO, by free slots and HBM bytes
                while waiting:
                    s = waiting[0]
                    slots_full = len(active) + in_setup >= self.max_slots
                    if slots_full or reserved + s.nbytes > self.budget:
                        s.waited = True
                        if not slots_full:
                            s.waited_bytes = True
                        break
                    waiting.popleft()
                    reserved += s.nbytes
                    peak_reserved = max(peak_reserved, reserved)
                    s.admitted_at = t
                    s.t_request = s.arrival
                    in_setup += 1
                    with lock:
                        setup_q.append(s)
                        lock.notify()
                # sessions whose setup finished join the active set
                with lock:
                    while setup_done:
                        active.append(setup_done.popleft())
                        in_setup -= 1
                peak_active = max(peak_active, len(active))
                # launch every ready build; collect completions
                progressed = False
                for s in list(active):
                    stop_now = self._cancelled(s, now())
                    if s.token is None:
                        if stop_now:  # nothing on the GPU: release at once
                            self.engine.close(s)
                            s.state = None
                            reserved -= s.nbytes
                            active.remove(s)
                            s.cancelled = True
                            cancelled.append(s)
                        else:
                            s.token = self.engine.launch(s)
                        progressed = True
                    elif self.engine.done(s.token):
                        tdone = now()
                        s.latencies.append(tdone - s.t_request)
                        if self.capture:
                            s.results.append(self.engine.result(s))
                        s.it += 1
                        s.token = None
                        progressed = True
                        if stop_now and s.it < s.niter:  # the build in flight has finished
                            self.engine.close(s)
                            s.state = None
                            reserved -= s.nbytes
                            active.remove(s)
                            s.cancelled = True
                            cancelled.append(s)
                        elif s.it >= s.niter:
                            self.engine.close(s)
                            s.state = None
                            reserved -= s.nbytes
                            active.remove(s)
                            finished.append(s)
                        else:
                            self.engine.advance(s)
                            s.t_request = tdone
                            s.token = self.engine.launch(s)
                if not progressed:
                    time.sleep(self.poll_s)
        finally:
            with lock:
                stop[0] = True
                lock.notify_all()
            for th in ths:
                th.join()
        wall = now()
        lat = np.array([x for s in finished for x in s.latencies]) * 1e3
        nb = int(lat.size)
        finished.sort(key=lambda s: s.sid)
        report = {
            "sessions": len(finished), "builds": nb, "wall_s": round(wall, 3),
            "builds_per_s": round(nb / wall, 2) if wall > 0 else None,
            "latency_ms_p50": round(float(np.percentile(lat, 50)), 3) if nb else None,
            "latency_ms_p99": round(float(np.percentile(lat, 99)), 3) if nb else None,
            "latency_ms_mean": round(float(lat.mean()), 3) if nb else None,
            "peak_reserved_bytes": int(peak_reserved), "hbm_budget_bytes": self.budget,
            "peak_concurrent_sessions": int(peak_active), "sessions_that_waited": int(sum(s.waited for s in finished)),
            "sessions_waited_for_bytes": int(sum(s.waited_bytes for s in finished + cancelled)),
            "cancelled": len(cancelled),
            "setup_ms_mean": round(1e3 * float(np.mean([s.ready_at - s.admitted_at for s in finished])), 3)
            if finished else None,
        }
        return report, finished


class LiberiEngine(Engine):
    """Sessions on the CUDA engine: one handle, stream, packed D and F per
    session; builds enqueued with liberi_c_fock_build_device; the density of
    build i+1 is D_i plus seeded symmetric noise of `noise` (packed)."""

    def __init__(self, device=0, precision=1, fp32_cut=1e-7, schwarz_cut=1e-10, noise=1e-3):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.device = device
        self.precision = precision
        self.fp32_cut = fp32_cut
        self.schwarz_cut = schwarz_cut
        self.noise = noise
        self._bytes = {}  # per Schwarz table object: sessions of one pool molecule share it

    def bytes_needed(self, basis):
        from . import liberi
        key = id(basis["schwrz"])
        if key not in self._bytes:
            n = basis["num_bas"]
            self._bytes[key] = (liberi.setup_bytes(basis, self.schwarz_cut) + 2 * 8 * (n * (n + 1) // 2),
                                basis["schwrz"])
        return self._bytes[key][0]

    def open(self, s):
        from . import liberi
        from . import molecules as M
        torch = self.torch
        torch.cuda.set_device(self.device)
        b = s.basis
        if "schwrz" not in b:
            b["schwrz"] = liberi.schwarz(b)
        h = liberi.liberi_create()
        h.set_option("device", self.device)
        h.set_option("schwarz_cut", self.schwarz_cut)
        h.set_option("precision", self.precision)
        h.set_option("fp32_cut", self.fp32_cut)
        # concurrent sessions fill the GPU: no multi-stream spread of one build
        h.set_option("fan", 0)
        liberi.setup_from_basis(h, b)
        stream = torch.cuda.Stream(device=self.dev)
        D0 = s.D0 if s.D0 is not None else M.density(b["num_bas"], M.nocc_of(b), seed=s.seed)
        with torch.cuda.stream(stream):
            D = torch.from_numpy(D0).to(self.dev, non_blocking=False)
            F = torch.zeros_like(D)
        gen = torch.Generator(device=self.dev)
        stream.synchronize()
        return {"h": h, "stream": stream, "D": D, "F": F, "gen": gen}

    def launch(self, s):
        from . import liberi
        st = s.state
        liberi.fock_build_device(st["h"], st["D"].data_ptr(), st["F"].data_ptr(), st["stream"].cuda_stream)
        ev = self.torch.cuda.Event()
        ev.record(st["stream"])
        return ev

    def done(self, token):
        return token.query()

    def result(self, s):
        return s.state["F"].cpu().numpy().copy()

    def advance(self, s):
        torch = self.torch
        st = s.state
        st["gen"].manual_seed(int(s.seed) * 1000003 + s.it)
        with torch.cuda.stream(st["stream"]):
            st["D"].add_(self.noise * torch.randn(st["D"].shape, generator=st["gen"], device=self.dev,
                                                  dtype=torch.float64))

    def close(self, s):
        from . import liberi
        st = s.state
        st["stream"].synchronize()
        liberi.liberi_destroy(st["h"])
        st.clear()

    def density_sequence(self, s):
        """The densities session `s` sees (for isolation checks): list of
        host arrays, one per build."""
        from . import molecules as M
        torch = self.torch
        b = s.basis
        D0 = s.D0 if s.D0 is not None else M.density(b["num_bas"], M.nocc_of(b), seed=s.seed)
        D = torch.from_numpy(D0).to(self.dev)
        gen = torch.Generator(device=self.dev)
        out = [D.cpu().numpy().copy()]
        for it in range(1, s.niter):
            gen.manual_seed(int(s.seed) * 1000003 + it)
            D = D + self.noise * torch.randn(D.shape, generator=gen, device=self.dev, dtype=torch.float64)
            out.append(D.cpu().numpy().copy())
        return out


def poisson_sessions(pool, rate_builds, nsessions, niter=15, seed=0, densities=None):
    """Sessions drawn from `pool` (list of bases) arriving as a Poisson
    process whose build rate is `rate_builds` (sessions at rate/niter).
    `densities[k]`, when given, is the initial density sent with every
    session of pool molecule k (client-side data, made before serving)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(nsessions):
        t += rng.exponential(niter / rate_builds)
        k = int(rng.integers(0, len(pool)))
        out.append(Session(sid=i, basis=dict(pool[k]), niter=niter, seed=1000 + i, arrival=t,
                           D0=None if densities is None else densities[k]))
    return out
