#!/usr/bin/env python
"""Benchmark: RHF two-electron Fock build of a C60-shaped molecule in a
6-31G(d)-shaped basis (900 functions) on B200.

One step = one full Fock build (all 21 s/p/d quartet classes, FP64) over the
device-resident density, as libERI's liberi_fock_build / compute_integrals
does per SCF iteration.  Inputs are seeded synthetic data: C60 truncated
icosahedron with 2.65/2.74 bohr bonds, per-shell log-uniform exponents in
[0.1, 3000], D = 2 C C^T with 180 orthonormal random columns, Schwarz cut
1e-10 (the Schwarz table comes from the engine's own generator).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (under torchrun, one process per GPU): every rank builds a cost-balanced
slice of the quartets into a private packed F, and one NCCL all-reduce sums
F; the metric is ms per complete build (strong scaling).
`--impl reference` times the reference algorithm's CPU restatement (oracle/,
OpenMP on all host cores): one complete build of the same inputs (`value`),
then bounded samples of the quartets as its timed steps.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "C60 6-31G(d) Fock build ms"
SCHWARZ_CUT = 1e-10
MIXED_CUT = 1e-7          # serving loop (its configured cut)
BATCH_MIXED_CUT = 1e-5    # batched mixed tier: the loosest cut of the configured sweep
L2_FLUSH_BYTES = 512 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of oracle work for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-molecule batched SCF section")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop section")
    ap.add_argument("--no-fshells", action="store_true", help="skip the f-shell workload section")
    ap.add_argument("--serve-rates", type=str, default="10,20,50,100,200,500",
                    help="Poisson build-request rates (req/s) of the serving capacity curve; the configured "
                         "50-500 and two rates below the GPU's capacity for this pool")
    ap.add_argument("--serve-sessions", type=int, default=40,
                    help="SCF sessions (15 builds each) served per rate (half of it below 50 req/s)")
    return ap.parse_args()


def workload():
    from gms_liberi_b200 import molecules as M
    b = M.c60()
    return b, M.density(b["num_bas"], 180, seed=0)


def config(n):
    return {"workload": "C60 truncated icosahedron, 6-31G(d)-shaped basis (360 shells, 900 functions), "
                        "RHF two-electron Fock build, Schwarz cut 1e-10",
            "natoms": 60, "num_bas": 900, "nocc": 180, "schwarz_cut": SCHWARZ_CUT,
            "l2": "flushed between timed steps (512 MB device write outside the step events)",
            "parallelism": "single GPU" if n == 1 else ("quartets split across %d ranks in cost-balanced slices, NCCL all-reduce of packed F" % n)}


# ------------------------------------------------------------------ reference arm
def oracle_sampled_ms(basis, D, mod, seed=0, nthreads=0):
    """One oracle build over a hashed uniform 1/mod sample of every class's
    screened quartets (whole bra pairs).  Per class the full-run estimate is
    the candidate-enumeration wall time (paid once in a full run) plus the
    measured evaluation time scaled by screened / evaluated quartets.
    Returns (extrapolated ms, wall s, info)."""
    from oracle import oracle
    t0 = time.time()
    _, c, (tw, te, nth) = oracle.fock_build(basis, D, schwarz_cut=SCHWARZ_CUT, sample_mod=mod,
                                            sample_seed=seed, nthreads=nthreads, return_times=True)
    wall = time.time() - t0
    if mod == 1:
        ms = float(tw.sum() * 1e3)
    else:
        mean_q = te.sum() / max(int(c[:, 3].sum()), 1)
        ms = 0.0
        for k in range(21):
            if c[k, 0] == 0:
                continue
            enum = max(tw[k] - te[k] / nth, 0.0)
            ev = te[k] / nth * c[k, 0] / c[k, 3] if c[k, 3] > 0 else mean_q / nth * c[k, 0]
            ms += (enum + ev) * 1e3
    return ms, wall, {"sample_mod": mod, "evaluated_quartets": int(c[:, 3].sum()),
                      "screened_quartets": int(c[:, 0].sum()), "seconds": round(wall, 2), "threads": nth}


def oracle_extrapolated_ms(basis, D, budget_s, seed=0, nthreads=0):
    """oracle_sampled_ms with the sample sized to about budget_s seconds of
    wall time by a small pilot sample.  Returns (ms, info)."""
    from oracle import oracle
    _, c0, (tw, te, nth) = oracle.fock_build(basis, D, schwarz_cut=SCHWARZ_CUT, sample_mod=20000,
                                             sample_seed=seed + 1000, nthreads=nthreads, return_times=True)
    per_q = te.sum() / max(int(c0[:, 3].sum()), 1)  # thread-seconds per evaluated quartet
    mod = int(np.clip(per_q * c0[:, 0].sum() / (budget_s * nth), 1, 2000000))
    for attempt in range(2):
        ms, wall, info = oracle_sampled_ms(basis, D, mod, seed=seed, nthreads=nthreads)
        # the small pilot overstates the per-quartet cost: resize the sample
        # once when it ran well short of the budget
        if attempt or mod == 1 or wall >= 0.5 * budget_s:
            break
        mod = max(1, int(mod * wall / budget_s))
    return ms, info


def run_reference(args):
    """The reference algorithm's CPU restatement (oracle/, OpenMP on every host
    core) on the same C60 inputs.  No library of this repository is loaded:
    the Schwarz table is the oracle's own, computed before any timing.
    `value` is one complete, unsampled build, timed by the host clock (the
    reference's bench_c60.F90:190-192 times its build the same way); the K
    timed steps (after W warm-up steps) are hashed 1/M samples of every
    class's screened quartets, each extrapolated per class by exact counts,
    so that the whole run stays within a few minutes; `ms_per_step` is their
    measured wall time per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle
    oracle.lib()
    basis, D = workload()
    basis["schwrz"] = oracle.schwarz(basis)
    cores = os.cpu_count()
    t0 = time.time()
    _, full = oracle.fock_build(basis, D, schwarz_cut=SCHWARZ_CUT, nthreads=cores, return_info=True)
    full_ms = (time.time() - t0) * 1e3
    # steps of about 3 s each (90 s over the default 20 + 5): the sample size
    # follows from the measured complete build
    per_step = max(2.0, min(8.0, 90.0 / max(1, args.steps + args.warmup)))
    mod = int(max(1, round(full_ms / 1e3 / per_step)))
    walls, extrap = [], []
    info = None
    for s in range(args.warmup + args.steps):
        ms, wall, info = oracle_sampled_ms(basis, D, mod, seed=s, nthreads=cores)
        if s >= args.warmup:
            walls.append(wall * 1e3)
            extrap.append(ms)
    step_ms = float(np.mean(walls))
    v = full_ms
    sample = ("value: one complete unsampled build (%d screened quartets, %.1f s wall); steps: a hashed uniform "
              "1/%d sample of each class's screened quartets per step (%d of %d), extrapolated per class by exact "
              "counts to %.0f ms (mean over steps); reference algorithm restated in C (oracle/), OpenMP over "
              "quartets" % (int(full["counts"][:, 0].sum()), full_ms / 1e3, info["sample_mod"],
                            info["evaluated_quartets"], info["screened_quartets"], float(np.mean(extrap))))
    line = {"metric": METRIC, "value": round(v, 3), "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(step_ms, 3), "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config(1),
            "cpu_baseline": {"value": round(v, 3), "unit": "ms", "cores": cores, "kind": "port", "sample": sample},
            "full_build_ms": round(full_ms, 1),
            "sampled_steps": {"ms_wall_per_step": round(step_ms, 1), "sample_mod": info["sample_mod"],
                              "extrapolated_ms_mean": round(float(np.mean(extrap)), 1),
                              "extrapolated_ms_min": round(float(np.min(extrap)), 1),
                              "extrapolated_ms_max": round(float(np.max(extrap)), 1)},
            "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.lines = []
        self.proc = None
        cmd = ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "200"]
        if uuid:
            cmd += ["-i", uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_per_launch(kernel):
    """dram bytes per launch of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "%s_c60.txt" % kernel)
    if not os.path.exists(path):
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def run_ours(args):
    import torch
    from gms_liberi_b200 import flops, liberi, ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    basis, Dh = workload()
    basis["schwrz"] = liberi.schwarz(basis)
    h = liberi.liberi_create()
    h.set_option("device", local)
    h.set_option("schwarz_cut", SCHWARZ_CUT)
    if world > 1:
        h.set_option("rank_split", 1)  # cost-balanced slices: the same F, even time per GPU
    liberi.setup_from_basis(h, basis, my_rank=rank, num_procs=world)
    st0 = h.stats()
    ntri = Dh.size
    D = torch.from_numpy(Dh).to(dev)
    F = torch.zeros(ntri, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    # a dedicated stream: the engine's kernels, the flush, the copies, the
    # all-reduce and the timing events are all ordered on it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    launched = int(sum(1 for k in range(21) if st0["quartets"][k] > 0))

    def partial(r, n):
        liberi.fock_build_device(h, D.data_ptr(), F.data_ptr(), stream.cuda_stream)
        return F

    def step():
        ranks.reduced_fock(partial)  # one NCCL all-reduce of the packed F when N > 1

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_loop(nsteps, per_class=False):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        cls = np.zeros(21)
        barrier()
        for s in range(nsteps):
            flush.zero_()
            ev[s][0].record(stream)
            step()
            ev[s][1].record(stream)
            if per_class:
                cls += h.stats()["kernel_ms"][:21]  # the s/p/d classes (C60 has no f shells)
        barrier()
        ms = [a.elapsed_time(b) for a, b in ev]
        return float(np.mean(ms)), cls / max(1, nsteps)

    def max_over_ranks(x):
        return ranks.max_over_ranks(x, device=dev)

    assert stream.cuda_stream != 0
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass

    # warm-up, then the timed region (clocks sampled, per-class events on)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clk = ClockSampler(uuid)
    ms_local, _ = timed_loop(args.steps)
    clocks = clk.stop()
    ms = max_over_ranks(ms_local)
    F_fp64 = F.detach().clone()
    # per-class device times (events around each class; the classes then run
    # on one stream): the roofline figures of the dominant kernel
    h.set_option("timing", 1)
    _, cls_ms = timed_loop(max(3, args.steps // 2), per_class=True)
    h.set_option("timing", 0)

    # roofline of the dominant class kernel: numerator = operations of the
    # reference algorithm (flop_constants.json, the oracle's op-counting
    # build); the engine's own arithmetic as a second figure
    k_dom = int(np.argmax(cls_ms))
    kname = liberi.KERNELS[k_dom]
    npq, nsq = int(st0["prim_quartets"][k_dom]), int(st0["quartets"][k_dom])
    fl = flops.class_flops(k_dom, npq, nsq)
    fl_eng = flops.engine_class_flops(k_dom, npq, nsq)
    peak_fp64 = liberi.microbench(0)
    t_dom = cls_ms[k_dom] * 1e-3
    achieved = fl / t_dom / 1e12
    build_tf = flops.build_flops(st0) / (ms_local * 1e-3) / 1e12
    build_tf_eng = flops.engine_build_flops(st0) / (ms_local * 1e-3) / 1e12
    roofline = {"bound": "fp64", "kernel": "class_kernel<%s>" % kname, "achieved": round(achieved, 3),
                "peak": round(peak_fp64, 3), "unit": "TFLOP/s", "frac": round(achieved / peak_fp64, 4),
                "numerator": "operations of the reference algorithm per primitive and shell quartet "
                             "(gms_liberi_b200/flop_constants.json, oracle op-counting build) x exact counts",
                "peak_source": "measured FP64 FMA throughput on this GPU (liberi_c_microbench 0); "
                               "MEASURED_PEAKS.json carries no FP64 figure",
                "traffic": traffic_per_launch(kname), "share": round(float(cls_ms[k_dom] / cls_ms.sum()), 3),
                "engine_count": {"achieved": round(fl_eng / t_dom / 1e12, 3),
                                 "frac": round(fl_eng / t_dom / 1e12 / peak_fp64, 4),
                                 "note": "the engine's own arithmetic (gms_liberi_b200/flops.py engine_costs)"},
                "build_achieved_tflops": round(build_tf, 3), "build_achieved_tflops_engine_count": round(build_tf_eng, 3),
                "per_class_ms": {liberi.KERNELS[k]: round(float(cls_ms[k]), 3) for k in range(21)}}

    # end to end through the public API with host buffers
    pin_D = torch.from_numpy(Dh).pin_memory()
    pin_F = torch.zeros(ntri, dtype=torch.float64).pin_memory()
    e2e_vals = []
    if world == 1:
        Fh = pin_F.numpy()
        Dp = pin_D.numpy()
        for s in range(args.warmup + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            # host clock around the public call (H2D of D, build, D2H of F,
            # synchronous): everything a caller waits for
            t0 = time.perf_counter()
            liberi.liberi_fock_build(h, Dp, Fh, ntri)  # host buffers, the handle's own stream
            t1 = time.perf_counter()
            if s >= args.warmup:
                e2e_vals.append((t1 - t0) * 1e3)
        e2e_ms = float(np.mean(e2e_vals))
    else:
        ev = []
        barrier()
        for s in range(args.warmup + args.steps):
            flush.zero_()
            a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            D.copy_(pin_D, non_blocking=True)
            step()
            pin_F.copy_(F, non_blocking=True)
            b2.record(stream)
            if s >= args.warmup:
                ev.append((a, b2))
        barrier()
        e2e_ms = max_over_ranks(float(np.mean([a.elapsed_time(b2) for a, b2 in ev])))

    # mixed precision at the serving cut, and the accuracy sweep of config 3
    mixed = None
    if not args.no_mixed:
        h.set_option("precision", 1)
        sweep = []
        mixed_roofline = None
        peak_fp32 = liberi.microbench(1)
        # the configured sweep is 1e-5..1e-8; 1e-2..1e-4 are added to
        # locate the loosest cut that still meets |dE| <= 1e-6 Eh
        for cut in (1e-2, 1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8):
            h.set_option("fp32_cut", cut)
            for _ in range(2):
                step()
            m_ms = max_over_ranks(timed_loop(max(3, args.steps // 2))[0])
            st_m = h.stats()
            f32 = float(st_m["fp32_quartets"].sum()) / max(1.0, float(st_m["quartets"].sum()))
            dF = (F - F_fp64).abs().max().item()
            dE = 0.5 * abs(float(torch.dot(F - F_fp64, _weights(D))))
            sweep.append({"fp32_cut": cut, "ms": round(m_ms, 3), "speedup_vs_fp64": round(ms / m_ms, 3),
                          "fp32_quartet_share": round(f32, 4),
                          "max_dF_vs_fp64": dF, "dE_vs_fp64": dE})
            if cut == 1e-5:
                # FP32+FP64 roofline of the mixed build: the time the reference-
                # algorithm operations would take at the measured FP64 and FP32
                # peaks (each class's operations split between the tiers by its
                # FP32 quartet share) over the measured time
                t_ideal = 0.0
                for k in range(21):
                    q = float(st_m["quartets"][k])
                    if q <= 0:
                        continue
                    s32 = float(st_m["fp32_quartets"][k]) / q
                    w = flops.class_flops(k, int(st0["prim_quartets"][k]), int(st0["quartets"][k]))
                    t_ideal += w * (1.0 - s32) / (peak_fp64 * 1e12) + w * s32 / (peak_fp32 * 1e12)
                mixed_roofline = {"fp32_cut": cut, "ideal_ms": round(t_ideal * 1e3, 3), "ms": round(m_ms, 3),
                                  "frac": round(t_ideal * 1e3 / m_ms, 4), "peak_fp64_tflops": round(peak_fp64, 3),
                                  "peak_fp32_tflops": round(peak_fp32, 3),
                                  "note": "reference-algorithm operations; tiers split by FP32 quartet share"}
        h.set_option("precision", 0)
        ok = [s for s in sweep if s["dE_vs_fp64"] <= 1e-6]
        best = max(ok, key=lambda s: s["speedup_vs_fp64"]) if ok else None
        conf = [s for s in ok if 1e-8 <= s["fp32_cut"] <= 1e-5]
        best_conf = max(conf, key=lambda s: s["speedup_vs_fp64"]) if conf else None
        mixed = {"reference_path": "plain FP64 GPU build (parity-tested against the oracle: max|dF| 3e-12, "
                                   "|dE| < 1e-11 on this workload)",
                 "fp32_prim": h.get_option("fp32_prim"),
                 "best_in_configured_sweep_1e-5_1e-8": best_conf, "best_within_dE_1e-6": best,
                 "roofline_fp32_fp64": mixed_roofline, "sweep": sweep}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count()
        cpu_ms, info = oracle_extrapolated_ms(basis, Dh, args.cpu_budget, nthreads=cores)
        cpu = {"value": round(cpu_ms, 1), "unit": "ms", "cores": cores, "kind": "port",
               "sample": "hashed uniform 1/%d sample of each class's screened quartets (%d of %d), "
                         "%.1f s wall on %d threads, extrapolated per class by exact counts"
                         % (info["sample_mod"], info["evaluated_quartets"], info["screened_quartets"],
                            info["seconds"], info["threads"])}

    batched = None
    if world == 1 and not args.no_batched:
        # the batched configuration splits its work between the FP64 and the
        # mixed-precision tiers: the same 256-molecule SCF run in each
        batched = {"fp64": run_batched(dev, stream, 0), "mixed": run_batched(dev, stream, 1)}
        e64, emx = batched["fp64"].pop("_energies"), batched["mixed"].pop("_energies")
        batched["mixed"]["max_dE_vs_fp64_batch"] = float(np.abs(emx - e64).max())
        batched["mixed_speedup_vs_fp64_batch"] = round(batched["fp64"]["ms_per_iteration_graph"] /
                                                       batched["mixed"]["ms_per_iteration_graph"], 3)
    fshells = None
    if world == 1 and not args.no_fshells:
        fshells = run_fshells(dev, stream, cpu=not args.no_cpu_baseline)
    serve = None
    if world == 1 and not args.no_serve:
        curve = [run_serve(local, float(r), args.serve_sessions if float(r) >= 50 else max(1, args.serve_sessions // 2))
                 for r in args.serve_rates.split(",") if r]
        serve = {"curve": curve,
                 "summary": [{k: c[k] for k in ("rate_req_per_s", "builds_per_s", "latency_ms_p50", "latency_ms_p99",
                                                 "peak_device_bytes_measured", "peak_concurrent_sessions")}
                             for c in curve]}

    if rank == 0:
        line = {"metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded C60 geometry, 6-31G(d)-shaped exponents, D = 2CC^T)",
                "config": config(world), "clocks": clocks,
                "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 8 * ntri,
                        "d2h_bytes_per_step": 8 * ntri},
                "gpu_launches": launched * args.steps, "roofline": roofline, "cpu_baseline": cpu,
                "mixed": mixed, "batched": batched, "serve": serve, "f_shells": fshells,
                "quartets": int(st0["quartets"].sum()), "prim_quartets": int(st0["prim_quartets"].sum())}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    liberi.liberi_destroy(h)
    return 0


BATCH_MOLECULES = 256
BATCH_ITERATIONS = 15


def run_batched(dev, stream, precision=0):
    """Batched multi-molecule SCF iterations: 256 seeded molecules of 3-40
    atoms (C/N/O/H 3:1:1:5, 1.9 bohr minimum separation, 0.01 atoms/bohr^3),
    6-31G(d)-shaped basis, 15 Fock builds each with D perturbed by seeded
    symmetric noise of 1e-3 per iteration.  One iteration of all molecules is
    one captured CUDA graph (F zeroing + one launch per class over every
    molecule's tasks), after the per-class autotuner; the same iterations
    through 256 separate per-molecule builds are timed beside it."""
    import torch
    from gms_liberi_b200 import liberi
    from gms_liberi_b200 import molecules as M

    rng = np.random.default_rng(2024)
    natoms = rng.integers(3, 41, BATCH_MOLECULES)
    t0 = time.time()
    bases = [M.random_molecule(int(n), seed=i) for i, n in enumerate(natoms)]
    hs = []
    for b in bases:
        b["schwrz"] = liberi.schwarz(b)
        h = liberi.liberi_create()
        h.set_option("schwarz_cut", SCHWARZ_CUT)
        if precision == 1:
            h.set_option("precision", 1)
            h.set_option("fp32_cut", BATCH_MIXED_CUT)
        liberi.setup_from_basis(h, b)
        hs.append(h)
    setup_s = time.time() - t0
    ntri = [b["num_bas"] * (b["num_bas"] + 1) // 2 for b in bases]
    off = np.concatenate([[0], np.cumsum(ntri)])
    D0 = np.concatenate([M.density(b["num_bas"], M.nocc_of(b), seed=i) for i, b in enumerate(bases)])
    D_all = torch.from_numpy(D0).to(dev)
    F_all = torch.zeros_like(D_all)
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    noise = 1e-3 * torch.randn((BATCH_ITERATIONS, D_all.numel()), generator=g, device=dev, dtype=torch.float64)
    Dp = [D_all.data_ptr() + 8 * int(o) for o in off[:-1]]
    Fp = [F_all.data_ptr() + 8 * int(o) for o in off[:-1]]
    torch.cuda.synchronize()

    def iterations(one_iteration):
        D_all.copy_(torch.from_numpy(D0).to(dev))
        one_iteration()  # warm-up on the unperturbed density
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(BATCH_ITERATIONS)]
        D_all.copy_(torch.from_numpy(D0).to(dev))
        torch.cuda.synchronize()
        for it in range(BATCH_ITERATIONS):
            ev[it][0].record(stream)
            D_all.add_(noise[it])
            one_iteration()
            ev[it][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    def unbatched():
        for h, dp, fp in zip(hs, Dp, Fp):
            liberi.fock_build_device(h, dp, fp, stream.cuda_stream)

    ms_single = iterations(unbatched)
    F_single = F_all.clone()

    bt = liberi.Batch(hs)
    bt.bind(Dp, Fp)
    t0 = time.time()
    chunks = bt.autotune(reps=2)
    tune_s = time.time() - t0
    bt.capture()
    ms_graph = iterations(lambda: bt.launch(stream.cuda_stream))
    dF = float((F_all - F_single).abs().max().item())
    # two-electron energy of every molecule at the last iteration (the same
    # densities in both tiers: seeded noise)
    wD = []
    for b, o in zip(bases, off[:-1]):
        n = b["num_bas"]
        w = torch.full((n * (n + 1) // 2,), 2.0, dtype=torch.float64, device=dev)
        idx = torch.arange(1, n + 1, device=dev)
        w[idx * (idx + 1) // 2 - 1] = 1.0
        seg = slice(int(o), int(o) + w.numel())
        wD.append(0.5 * float(torch.dot(w * D_all[seg], F_all[seg])))
    energies = np.array(wD)
    n_classes = int(sum(1 for k in range(21) if any(h.stats()["quartets"][k] > 0 for h in hs)))
    bt.destroy()
    for h in hs:
        liberi.liberi_destroy(h)
    it_ms = float(np.mean(ms_graph))
    return {"molecules": BATCH_MOLECULES, "atoms": [int(natoms.min()), int(natoms.max())],
            "functions": [int(min(b["num_bas"] for b in bases)), int(max(b["num_bas"] for b in bases)),
                          int(sum(b["num_bas"] for b in bases))],
            "iterations": BATCH_ITERATIONS,
            "dtype": "f64" if precision == 0 else "mixed f32/f64, fp32_cut %g" % BATCH_MIXED_CUT,
            "ms_per_iteration_graph": round(it_ms, 3),
            "ms_per_iteration_p50": round(float(np.median(ms_graph)), 3),
            "ms_per_iteration_separate_builds": round(float(np.mean(ms_single)), 3),
            "speedup_vs_separate_builds": round(float(np.mean(ms_single)) / it_ms, 3),
            "builds_per_s": round(BATCH_MOLECULES / (it_ms * 1e-3), 1),
            "launches_per_iteration": 1 + n_classes,
            "max_dF_batched_vs_separate": dF,
            "autotune_kets_per_task": {liberi.KERNELS[k]: int(chunks[k]) for k in range(21) if chunks[k]},
            "autotune_s": round(tune_s, 2), "setup_s": round(setup_s, 2),
            "timing": "CUDA events per iteration (D update + build), inputs resident, no L2 flush "
                      "(all molecules' data fits in L2 as it would across SCF iterations)",
            "_energies": energies}


def run_fshells(dev, stream, cpu=True):
    """The f-shell classes on a 30-atom C/N/O/H cluster with a d and an f
    polarisation shell on every heavy atom and a p shell on every H (470
    functions; FP64, Schwarz table from the device generator, cut 1e-10),
    device-resident D/F, CUDA events on the build's stream, median of 5 builds
    after 2 (the working set stays in L2 between builds).  cpu_baseline: one
    complete oracle build of the same inputs on every host core."""
    import torch
    from gms_liberi_b200 import liberi
    from gms_liberi_b200 import molecules as M
    b = M.f_cluster(30, seed=5)
    b["schwrz"] = liberi.schwarz(b)
    D = M.density(b["num_bas"], M.nocc_of(b), seed=1)
    n = b["num_bas"]
    ntri = n * (n + 1) // 2
    dD = torch.tensor(D, device=dev)
    dF = torch.zeros(ntri, dtype=torch.float64, device=dev)
    h = liberi.liberi_create()
    h.set_option("schwarz_cut", SCHWARZ_CUT)
    liberi.setup_from_basis(h, b)
    ts = []
    for it in range(7):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        liberi.fock_build_device(h, dD.data_ptr(), dF.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= 2:
            ts.append(e0.elapsed_time(e1))
    st = h.stats()
    liberi.liberi_destroy(h)
    ms = float(np.median(ts))
    out = {"workload": "30-atom C/N/O/H cluster, 6-31G(d)-shaped s/p with one d and one f polarisation shell per "
                       "heavy atom and a p shell per H (polarisation exponents in [0.3, 3]), Schwarz cut 1e-10",
           "functions": n, "dtype": "f64", "ms": round(ms, 3),
           "quartets_spd": int(st["quartets"][:21].sum()), "quartets_f": int(st["quartets"][21:].sum()),
           "prim_quartets_f": int(st["prim_quartets"][21:].sum()),
           "timing": "CUDA events, median of 5 builds after 2, no L2 flush (working set L2-resident)"}
    if cpu:
        from oracle import oracle
        t0 = time.time()
        _, info = oracle.fock_build(b, D, schwarz_cut=SCHWARZ_CUT, nthreads=os.cpu_count(), return_info=True)
        wall = time.time() - t0
        out["cpu_baseline"] = {"value": round(wall * 1e3, 1), "unit": "ms", "cores": int(info["nthreads"]),
                               "kind": "port", "sample": "one complete build of the same inputs",
                               "f_classes_ms": round(float(info["t_wall"][21:].sum()) * 1e3, 1)}
        out["speedup_vs_cpu_baseline"] = round(wall * 1e3 / ms, 1)
    return out


_SERVE_POOL = None


def run_serve(local, rate, nsessions):
    """Serving loop: SCF sessions (15 Fock builds each, D perturbed by 1e-3
    seeded noise between builds) of molecules drawn from a seeded pool of
    10-200-atom molecules (C/N/O/H 3:1:1:5, 6-31G(d)-shaped), arriving as a
    Poisson process of `rate` build requests per second; mixed precision at
    cut 1e-7; admission by exact device bytes against 90% of the free HBM."""
    import torch
    from gms_liberi_b200 import liberi
    from gms_liberi_b200 import molecules as M
    from gms_liberi_b200.serve import FockServer, LiberiEngine, poisson_sessions

    global _SERVE_POOL
    if _SERVE_POOL is None:  # the same seeded pool for every rate of the curve
        rng = np.random.default_rng(77)
        pool = []
        for i, n in enumerate(rng.integers(10, 201, 8)):
            b = M.random_molecule(int(n), seed=500 + i)
            b["schwrz"] = liberi.schwarz(b)
            pool.append(b)
        dens = [M.density(b["num_bas"], M.nocc_of(b), seed=900 + k) for k, b in enumerate(pool)]
        _SERVE_POOL = (pool, dens)
    pool, dens = _SERVE_POOL
    sessions = poisson_sessions(pool, rate, nsessions, niter=15, seed=5, densities=dens)
    free0, total = torch.cuda.mem_get_info(local)
    peak = [0]
    stop = threading.Event()

    def sample():
        while not stop.is_set():
            f, _ = torch.cuda.mem_get_info(local)
            peak[0] = max(peak[0], free0 - f)
            time.sleep(0.02)

    th = threading.Thread(target=sample, daemon=True)
    th.start()
    eng = LiberiEngine(device=local, precision=1, fp32_cut=1e-7, schwarz_cut=SCHWARZ_CUT)
    srv = FockServer(eng, hbm_budget=int(0.9 * free0), max_slots=64)
    rep, done = srv.run(sessions)
    stop.set()
    th.join()
    rep.update({"rate_req_per_s": rate, "niter": 15, "precision": "mixed, fp32_cut 1e-7",
                "pool_atoms": sorted(int(len(b["symbols"])) for b in pool),
                "pool_functions": sorted(int(b["num_bas"]) for b in pool),
                "peak_device_bytes_measured": int(peak[0]),
                "latency": "per build, request (session arrival / previous build done) to F complete, "
                           "host clock; sessions run on their own streams and overlap"})
    return rep


def _weights(D):
    import torch
    n = int((np.sqrt(8 * D.numel() + 1) - 1) / 2)
    w = torch.full_like(D, 2.0)
    idx = torch.arange(1, n + 1, device=D.device)
    w[idx * (idx + 1) // 2 - 1] = 1.0
    return w * D


def main():
    args = parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
