"""Serving loop on the GPU: sessions of different molecules admitted while
others are in flight, builds overlapping on separate streams; every build's F
in the mix equals the same session's F computed alone (same densities, same
mixed-precision settings; only the order of FP64 atomics differs), and the
admission figure equals what setup allocates."""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from gms_liberi_b200.serve import FockServer, LiberiEngine, Session
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_SAME = 1e-10  # same session alone vs in the mix, mixed precision at cut 1e-7


def _pool():
    pool = [M.h2o_like(), M.ethane(), M.random_molecule(6, seed=11), M.random_molecule(9, seed=11)]
    for b in pool:
        b["schwrz"] = oracle.schwarz(b)
    return pool


def test_results_same_alone_and_in_the_mix():
    pool = _pool()
    sessions = [Session(sid=i, basis=dict(pool[i % len(pool)]), niter=3, seed=50 + i, arrival=0.002 * i)
                for i in range(7)]
    eng = LiberiEngine(precision=1, fp32_cut=1e-7, schwarz_cut=1e-10)
    srv = FockServer(eng, hbm_budget=8 << 30, max_slots=3, capture=True)
    rep, done = srv.run(sessions)
    assert rep["sessions"] == 7 and rep["builds"] == 21
    assert rep["peak_concurrent_sessions"] >= 2
    assert rep["sessions_that_waited"] >= 1  # 7 sessions, 3 slots
    for s in done:
        h = liberi.liberi_create()
        for k, v in (("schwarz_cut", 1e-10), ("precision", 1), ("fp32_cut", 1e-7)):
            h.set_option(k, v)
        liberi.setup_from_basis(h, s.basis)
        for it, D in enumerate(eng.density_sequence(s)):
            alone = liberi.fock(h, D)
            assert np.abs(s.results[it] - alone).max() <= TOL_SAME, (s.sid, it)
        liberi.liberi_destroy(h)


def test_admission_bytes_equal_setup_allocation():
    for b in _pool():
        h = liberi.liberi_create()
        h.set_option("schwarz_cut", 1e-10)
        liberi.setup_from_basis(h, b)
        assert liberi.setup_bytes(b, 1e-10) == h.stats()["device_bytes"]
        h.set_option("schwarz_cut", 1e-7)   # a re-plan keeps the figure exact
        liberi.fock(h, M.density(b["num_bas"], M.nocc_of(b)))
        assert liberi.setup_bytes(b, 1e-7) == h.stats()["device_bytes"]
        liberi.liberi_destroy(h)


def test_hbm_budget_holds_sessions_back_on_the_device():
    # slots are plentiful; the byte budget (room for the largest session and a
    # little more) is what makes sessions wait
    pool = _pool()
    eng = LiberiEngine(precision=1, fp32_cut=1e-7, schwarz_cut=1e-10)
    sizes = [eng.bytes_needed(b) for b in pool]
    budget = max(sizes) + min(sizes) // 2
    sessions = [Session(sid=i, basis=dict(pool[(i + 1) % len(pool)]), niter=2, seed=70 + i, arrival=0.0)
                for i in range(6)]
    srv = FockServer(eng, hbm_budget=budget, max_slots=64)
    rep, done = srv.run(sessions)
    assert rep["sessions"] == 6 and rep["builds"] == 12
    assert rep["sessions_waited_for_bytes"] >= 1
    assert rep["peak_reserved_bytes"] <= budget


def test_cancelled_session_releases_and_others_are_unaffected():
    pool = _pool()
    eng = LiberiEngine(precision=1, fp32_cut=1e-7, schwarz_cut=1e-10)
    sessions = [Session(sid=i, basis=dict(pool[i % len(pool)]), niter=4, seed=90 + i, arrival=0.0)
                for i in range(3)]
    srv = FockServer(eng, hbm_budget=8 << 30, max_slots=3, capture=True)
    srv.cancel(1)  # before its first build: never launches, releases at once
    rep, done = srv.run(sessions)
    assert rep["cancelled"] == 1 and rep["sessions"] == 2
    for s in done:
        h = liberi.liberi_create()
        for k, v in (("schwarz_cut", 1e-10), ("precision", 1), ("fp32_cut", 1e-7)):
            h.set_option(k, v)
        liberi.setup_from_basis(h, s.basis)
        for it, D in enumerate(eng.density_sequence(s)):
            assert np.abs(s.results[it] - liberi.fock(h, D)).max() <= TOL_SAME
        liberi.liberi_destroy(h)
