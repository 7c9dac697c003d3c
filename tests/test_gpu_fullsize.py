"""Full-size checks of the CUDA Fock build on the C60 6-31G(d)-shaped workload
(360 shells, 900 functions, Schwarz cut 1e-10), through the C ABI:
  * the screened-quartet set, class by class, equals the oracle's (exact
    counts; the oracle enumerates every candidate and evaluates a sample);
  * single classes against the oracle at full size, max|dF| <= 1e-10: every
    pair class (ss, sp, pp, sd, pd, dd) appears in at least one of them;
  * size-independent properties of the whole build: F is linear in D (the
    screening depends on Schwarz values and integrals, never on D), and the
    bilinear form sum_k D1_k F(D2)_k over the packed elements is symmetric in
    (D1, D2) by the permutational symmetry (ij|kl) = (kl|ij);
  * the mixed FP32/FP64 build within |dE| <= 1e-6 Eh of the FP64 build.
"""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from oracle import oracle

pytestmark = pytest.mark.gpu

CUT = 1e-10
TOL_F = 1e-10
# driver-order classes small enough for the oracle at full size
ORACLE_CLASSES = [0, 2, 6, 10, 11, 12, 13, 14, 15, 16, 18, 19, 20]


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


def build(h, D, **opts):
    old = {k: h.get_option(k) for k in opts}
    for k, v in opts.items():
        h.set_option(k, v)
    try:
        return liberi.fock(h, D), h.stats()
    finally:
        for k, v in old.items():
            h.set_option(k, v)


def test_screened_quartet_set_equals_oracle(c60):
    b, h, D, _ = c60
    _, cnt = oracle.fock_build(b, D, schwarz_cut=CUT, sample_mod=2000000, return_counts=True)
    _, st = build(h, D)
    assert (st["quartets"] == cnt[:, 0]).all(), (st["quartets"], cnt[:, 0])
    assert int(cnt[:, 0].sum()) == 264008469


@pytest.mark.parametrize("k", ORACLE_CLASSES)
def test_single_class_matches_oracle(c60, k):
    b, h, D, _ = c60
    Fo = oracle.fock_build(b, D, schwarz_cut=CUT, only_kernel=k)
    Fg, _ = build(h, D, class_mask=1 << k)
    assert np.abs(Fg - Fo).max() <= TOL_F, (liberi.KERNELS[k], np.abs(Fg - Fo).max())


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


def test_mixed_precision_energy_at_full_size(c60):
    _, h, D, _ = c60
    F64, _ = build(h, D)
    Fmx, st = build(h, D, precision=1, fp32_cut=1e-2)
    assert st["fp32_quartets"].sum() > 0.9 * st["quartets"].sum()
    assert abs(energy(D, Fmx) - energy(D, F64)) <= 1e-6
