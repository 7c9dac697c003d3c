"""Serving loop on the CPU: the scheduler of gms_liberi_b200.serve driven by a
fake engine whose builds take a fixed wall time, plus the library's host-only
footprint dry run (liberi_c_setup_bytes), which needs no device."""
import threading
import time

import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from gms_liberi_b200.serve import Engine, FockServer, Session, poisson_sessions
from oracle import oracle


class FakeEngine(Engine):
    """Builds complete `dur` seconds after launch; tracks resident bytes,
    live sessions and builds in flight."""

    def __init__(self, dur=0.004, setup=0.002):
        self.dur, self.setup = dur, setup
        self.lock = threading.Lock()
        self.resident = self.peak_resident = 0
        self.live = self.peak_live = 0
        self.inflight = self.peak_inflight = 0
        self.open_order = []

    def bytes_needed(self, basis):
        return basis["bytes"]

    def open(self, s):
        time.sleep(self.setup)
        with self.lock:
            self.resident += s.nbytes
            self.peak_resident = max(self.peak_resident, self.resident)
            self.live += 1
            self.peak_live = max(self.peak_live, self.live)
            self.open_order.append(s.sid)
        return {"D": 0}

    def launch(self, s):
        with self.lock:
            self.inflight += 1
            self.peak_inflight = max(self.peak_inflight, self.inflight)
        return [time.perf_counter() + self.dur, False]

    def done(self, tok):
        if not tok[1] and time.perf_counter() >= tok[0]:
            tok[1] = True
            with self.lock:
                self.inflight -= 1
        return tok[1]

    def result(self, s):
        return (s.sid, s.it, s.state["D"])

    def advance(self, s):
        s.state["D"] += 1

    def close(self, s):
        with self.lock:
            self.resident -= s.nbytes
            self.live -= 1


def _sessions(sizes, arrivals, niter=3):
    return [Session(sid=i, basis={"bytes": b}, niter=niter, seed=i, arrival=t)
            for i, (b, t) in enumerate(zip(sizes, arrivals))]


def test_every_build_completes_in_order():
    eng = FakeEngine()
    srv = FockServer(eng, hbm_budget=10_000, max_slots=8, capture=True)
    rep, done = srv.run(_sessions([100] * 5, [0.0, 0.001, 0.002, 0.01, 0.02], niter=4))
    assert rep["sessions"] == 5 and rep["builds"] == 20
    for s in done:
        assert len(s.latencies) == 4
        # each build saw the density of its own iteration
        assert [r[1] for r in s.results] == [0, 1, 2, 3]
        assert [r[2] for r in s.results] == [0, 1, 2, 3]
        assert all(l >= eng.dur * 0.9 for l in s.latencies)


def test_admission_respects_hbm_budget_and_slots():
    eng = FakeEngine()
    srv = FockServer(eng, hbm_budget=1000, max_slots=3)
    sizes = [400, 300, 500, 200, 100, 600, 250]
    rep, done = srv.run(_sessions(sizes, [0.0] * len(sizes)))
    assert rep["sessions"] == len(sizes)
    assert eng.peak_resident <= 1000 and rep["peak_reserved_bytes"] <= 1000
    assert eng.peak_live <= 3
    assert rep["sessions_that_waited"] >= 1
    # FIFO: a large session at the head is not overtaken by smaller ones
    # (admission order; set-ups then run on several worker threads)
    adm = [s.admitted_at for s in done]  # done is in session order
    assert adm == sorted(adm)


def test_builds_of_different_sessions_overlap():
    eng = FakeEngine(dur=0.01)
    srv = FockServer(eng, hbm_budget=10_000, max_slots=8)
    rep, _ = srv.run(_sessions([10] * 4, [0.0, 0.0, 0.005, 0.012], niter=5))
    assert eng.peak_inflight >= 3  # continuous batching, not one build at a time
    assert rep["peak_concurrent_sessions"] >= 3


def test_session_above_budget_is_rejected():
    srv = FockServer(FakeEngine(), hbm_budget=100)
    with pytest.raises(ValueError):
        srv.run(_sessions([50, 150], [0.0, 0.0]))


def test_poisson_arrivals_are_seeded_and_ordered():
    pool = [{"bytes": 1}, {"bytes": 2}]
    a = poisson_sessions(pool, rate_builds=100.0, nsessions=20, niter=15, seed=3)
    b = poisson_sessions(pool, rate_builds=100.0, nsessions=20, niter=15, seed=3)
    assert [s.arrival for s in a] == [s.arrival for s in b]
    t = np.array([s.arrival for s in a])
    assert (np.diff(t) > 0).all()
    # mean inter-arrival of sessions: niter / rate
    assert 0.05 < np.mean(np.diff(t)) < 0.3


def test_setup_bytes_dry_run():
    b = M.ethane()
    b["schwrz"] = oracle.schwarz(b)
    n_loose = liberi.setup_bytes(b, schwarz_cut=1e-6)
    n_tight = liberi.setup_bytes(b, schwarz_cut=1e-12)
    # tables, pair data, D and F are fixed; the plans shrink as the cut loosens
    assert 0 < n_loose < n_tight
    assert n_tight > 2 * 8 * (b["num_bas"] * (b["num_bas"] + 1) // 2)
    with pytest.raises(liberi.LiberiError):
        bad = dict(b)
        bad["ang_mom"] = [9] * b["nsh"]
        liberi.setup_bytes(bad)


def test_waits_for_hbm_bytes_not_slots():
    # plenty of slots: the second session is held back by the byte budget
    eng = FakeEngine(dur=0.005)
    srv = FockServer(eng, hbm_budget=1000, max_slots=64)
    rep, _ = srv.run(_sessions([700, 600, 100], [0.0, 0.0, 0.0]))
    assert rep["sessions"] == 3
    assert rep["sessions_waited_for_bytes"] >= 1
    assert eng.peak_resident <= 1000


def test_cancel_queued_session_is_never_set_up():
    eng = FakeEngine(dur=0.01)
    srv = FockServer(eng, hbm_budget=1000, max_slots=1)
    ss = _sessions([100, 100, 100], [0.0, 0.0, 0.0], niter=4)
    ss[2].cancel_at = 0.005  # still queued behind the single slot
    rep, done = srv.run(ss)
    assert rep["cancelled"] == 1 and rep["sessions"] == 2
    assert 2 not in eng.open_order
    assert eng.resident == 0 and eng.live == 0


def test_cancel_in_flight_session_finishes_its_build_and_releases():
    eng = FakeEngine(dur=0.02)
    srv = FockServer(eng, hbm_budget=1000, max_slots=4, capture=True)
    ss = _sessions([300, 300], [0.0, 0.0], niter=10)
    ss[0].cancel_at = 0.03  # during its second build
    rep, done = srv.run(ss)
    assert rep["cancelled"] == 1 and rep["sessions"] == 1
    assert done[0].sid == 1 and len(done[0].latencies) == 10
    # the cancelled session stopped after the build it had on the device
    assert 1 <= ss[0].it < 10 and ss[0].state is None
    assert eng.resident == 0 and eng.live == 0 and eng.inflight == 0


def test_cancel_from_another_thread():
    eng = FakeEngine(dur=0.01)
    srv = FockServer(eng, hbm_budget=1000, max_slots=2)
    ss = _sessions([100, 100, 100], [0.0, 0.0, 0.0], niter=20)
    t = threading.Timer(0.05, srv.cancel, args=(1,))
    t.start()
    rep, done = srv.run(ss)
    t.join()
    assert rep["cancelled"] == 1 and {s.sid for s in done} == {0, 2}
    assert eng.resident == 0
