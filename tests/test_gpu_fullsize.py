"""Full-size checks of the CUDA Fock build on the C60 6-31G(d)-shaped workload
(360 shells, 900 functions, 180 occupied columns, Schwarz cut 1e-10), through
the C ABI, against one full, unsampled oracle build of the same inputs (run
class by class on every host core, about a minute and a half on 16 threads;
the sum of the 21 class builds is the complete F):
  * the screened-quartet set of every class equals the oracle's: the count,
    sum and xor of a 64-bit hash of every quartet the class kernels walk;
  * every one of the 21 classes against the oracle, max|dF| <= 1e-10;
  * the complete F, max|dF| <= 1e-10, and E, |dE| <= 1e-9 Eh;
  * the mixed FP32/FP64 build at cuts inside the configured sweep
    (1e-5 ... 1e-8) within |dE| <= 1e-6 Eh of the oracle, with its per-build
    FP64 and FP32 task lists covering the same screened set;
  * size-independent properties of the whole build: F is linear in D (the
    screening depends on Schwarz values and integrals, never on D), and the
    bilinear form sum_k D1_k F(D2)_k over the packed elements is symmetric in
    (D1, D2) by the permutational symmetry (ij|kl) = (kl|ij);
  * the engine's own Schwarz generator gives the same screened set as the
    oracle's table (the inputs the benchmark builds from).
"""
import time

import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from oracle import oracle

pytestmark = pytest.mark.gpu

CUT = 1e-10
TOL_F = 1e-10
TOL_E = 1e-9
TOL_E_MIXED = 1e-6


def energy(D, F):
    n = int((np.sqrt(8 * D.size + 1) - 1) / 2)
    w = np.full(D.size, 2.0)
    w[np.arange(1, n + 1) * np.arange(2, n + 2) // 2 - 1] = 1.0
    return 0.5 * np.sum(w * D * F)


@pytest.fixture(scope="module")
def c60():
    b = M.c60()
    b["schwrz"] = oracle.schwarz(b)
    h = liberi.liberi_create()
    h.set_option("schwarz_cut", CUT)
    liberi.setup_from_basis(h, b)
    n = b["num_bas"]
    yield b, h, M.density(n, 180, seed=0), M.density(n, 180, seed=1)
    liberi.liberi_cleanup(h)
    liberi.liberi_destroy(h)


@pytest.fixture(scope="module")
def oracle_c60(c60):
    """The oracle's complete C60 build, class by class (no sampling)."""
    b, _, D, _ = c60
    t0 = time.time()
    per_class, fp = [], np.zeros((21, 3), dtype=np.uint64)
    nth = 0
    for k in range(21):
        Fk, info = oracle.fock_build(b, D, schwarz_cut=CUT, only_kernel=k, return_info=True)
        per_class.append(Fk)
        fp[k] = info["fingerprint"][k]
        nth = info["nthreads"]
    wall = time.time() - t0
    print("\noracle full C60 build: %.1f s on %d threads, %d screened quartets"
          % (wall, nth, int(fp[:, 0].astype(np.int64).sum())))
    return per_class, np.sum(per_class, axis=0), fp


def build(h, D, **opts):
    old = {k: h.get_option(k) for k in opts}
    for k, v in opts.items():
        h.set_option(k, v)
    try:
        F = liberi.fock(h, D)
        st = h.stats()
        st["fingerprint"] = h.quartet_fingerprint()
        return F, st
    finally:
        for k, v in old.items():
            h.set_option(k, v)


def test_screened_quartet_set_equals_oracle(c60, oracle_c60):
    _, h, D, _ = c60
    _, _, fp = oracle_c60
    _, st = build(h, D)
    assert (st["quartets"][:21] == fp[:, 0].astype(np.int64)).all(), (st["quartets"], fp[:, 0])
    bad = [liberi.KERNELS[k] for k in range(21) if not (st["fingerprint"][k] == fp[k]).all()]
    assert not bad, bad
    assert int(fp[:, 0].astype(np.int64).sum()) == 264008469


@pytest.mark.parametrize("k", range(21))
def test_single_class_matches_oracle(c60, oracle_c60, k):
    _, h, D, _ = c60
    per_class, _, _ = oracle_c60
    Fg, _ = build(h, D, class_mask=1 << k)
    err = np.abs(Fg - per_class[k]).max()
    assert err <= TOL_F, (liberi.KERNELS[k], err)


def test_full_build_matches_oracle(c60, oracle_c60):
    _, h, D, _ = c60
    _, Fo, _ = oracle_c60
    Fg, _ = build(h, D)
    dF = np.abs(Fg - Fo).max()
    dE = abs(energy(D, Fg) - energy(D, Fo))
    print("\nC60 FP64 vs oracle: max|dF| %.3e, |dE| %.3e Eh" % (dF, dE))
    assert dF <= TOL_F
    assert dE <= TOL_E


@pytest.mark.parametrize("fp32_cut", [1e-5, 1e-7])
def test_mixed_precision_against_oracle(c60, oracle_c60, fp32_cut):
    _, h, D, _ = c60
    _, Fo, fp = oracle_c60
    Fm, st = build(h, D, precision=1, fp32_cut=fp32_cut)
    assert st["fp32_quartets"].sum() > 0
    # the per-build FP64 and FP32 task lists partition the screened set
    assert (st["fingerprint"][:21] == fp).all()
    dE = abs(energy(D, Fm) - energy(D, Fo))
    print("\nC60 mixed cut %g vs oracle: max|dF| %.3e, |dE| %.3e Eh" % (fp32_cut, np.abs(Fm - Fo).max(), dE))
    assert dE <= TOL_E_MIXED


def test_engine_schwarz_gives_the_same_screened_set(c60, oracle_c60):
    b, _, D, _ = c60
    _, _, fp = oracle_c60
    b2 = dict(b)
    b2["schwrz"] = liberi.schwarz(b)
    h = liberi.liberi_create()
    h.set_option("schwarz_cut", CUT)
    liberi.setup_from_basis(h, b2)
    liberi.fock(h, D)
    got = h.quartet_fingerprint()
    liberi.liberi_destroy(h)
    assert (got[:21] == fp).all() and (got[21:] == 0).all()  # C60 has no f shells


def test_linear_in_density(c60):
    _, h, D1, D2 = c60
    F1, _ = build(h, D1)
    F2, _ = build(h, D2)
    F12, _ = build(h, D1 - 0.5 * D2)
    scale = max(1.0, np.abs(F1).max())
    assert np.abs(F12 - (F1 - 0.5 * F2)).max() <= 1e-11 * scale


def test_bilinear_form_symmetric(c60):
    _, h, D1, D2 = c60
    F1, _ = build(h, D1)
    F2, _ = build(h, D2)
    b12, b21 = float(np.dot(D1, F2)), float(np.dot(D2, F1))
    assert abs(b12 - b21) <= 1e-11 * max(1.0, abs(b12)), (b12, b21)
