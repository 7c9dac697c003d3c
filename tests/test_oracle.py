"""CPU oracle checks: the restatement against the reference's own known-answer
vectors (tests/fortran/test_*.F90, tol 1e-10), its Rys roots against exact
Boys-function moments, and the reference rank split."""
import numpy as np
import pytest
from scipy.special import gamma, gammainc

from oracle import oracle
from gms_liberi_b200 import molecules as M
from conftest import KAT_NAMES, load_kat


@pytest.mark.parametrize("name", KAT_NAMES)
def test_oracle_matches_reference_kat(name):
    d = load_kat(name)
    f = oracle.fock_build(d, d["density"])
    err = np.abs(f - d["fa_ref"]).max()
    assert err <= d["tol"], (name, err)


def _boys(m, T):
    if T < 1e-13:
        return 1.0 / (2 * m + 1)
    return gamma(m + 0.5) * gammainc(m + 0.5, T) / (2 * T ** (m + 0.5))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_oracle_rys_moments(n):
    # sum_i w_i u_i^k = F_k(T) for k < 2n (Gauss exactness of the Rys rule)
    for T in [0.0, 0.3, 2.0, 11.0, 24.9, 42.0, 54.9]:
        u, w = oracle.rys_roots(n, T, thr=60.0, rot=False)
        for k in range(2 * n):
            ex = _boys(k, T)
            assert abs(np.sum(w * u ** k) - ex) <= 5e-14 * ex + 1e-300, (n, T, k)


def test_oracle_asymptotic_branch():
    # rotated-axis classes switch to the large-T form for T > 25
    u, w = oracle.rys_roots(1, 30.0, thr=25.0, rot=True)
    assert abs(w[0] - 0.5 * np.sqrt(np.pi / 30.0)) < 1e-15
    assert abs(u[0] - 1.0 / 60.0) < 1e-15


@pytest.mark.parametrize("nsize", [2, 3, 7])
def test_oracle_rank_partials_sum_to_full(nsize):
    b = M.ethane()
    b["schwrz"] = oracle.schwarz(b)
    D = M.density(b["num_bas"], 9, seed=3)
    full = oracle.fock_build(b, D, schwarz_cut=1e-10)
    parts = sum(oracle.fock_build(b, D, schwarz_cut=1e-10, my_rank=r, num_procs=nsize) for r in range(nsize))
    assert np.abs(parts - full).max() < 1e-12


def test_rank_split_is_partition():
    # tile + rank arithmetic of int0000.F90:76-91 / int0001.F90:89-104 / int0101.F90:76-79
    for tile in range(4):
        for ntot in [1, 7, 100, 61237, 61238, 200000]:
            for nsize in [1, 2, 3, 7]:
                its = np.unique(np.linspace(1, ntot, min(ntot, 400)).astype(np.int64))
                for it in its:
                    owners = [r for r in range(nsize) if oracle.rank_owns(tile, ntot, int(it), r, nsize)]
                    assert len(owners) == 1, (tile, ntot, nsize, it, owners)


def test_oracle_screening_counts_monotone():
    b = M.ethane()
    b["schwrz"] = oracle.schwarz(b)
    D = M.density(b["num_bas"], 9)
    _, c1 = oracle.fock_build(b, D, schwarz_cut=1e-12, return_counts=True)
    _, c2 = oracle.fock_build(b, D, schwarz_cut=1e-8, return_counts=True)
    assert (c2[:, 0] <= c1[:, 0]).all() and c2[:, 0].sum() < c1[:, 0].sum()


def test_oracle_linear_and_symmetric_in_density():
    """The two properties the full-size GPU tests rest on, pinned on the
    oracle: F is linear in D, and sum_k D1_k F(D2)_k over the packed elements
    is symmetric in (D1, D2)."""
    b = M.ethane()
    b["schwrz"] = oracle.schwarz(b)
    n = b["num_bas"]
    D1, D2 = M.density(n, 9, seed=1), M.density(n, 9, seed=2)
    F1 = oracle.fock_build(b, D1, schwarz_cut=1e-10)
    F2 = oracle.fock_build(b, D2, schwarz_cut=1e-10)
    F12 = oracle.fock_build(b, D1 - 0.5 * D2, schwarz_cut=1e-10)
    assert np.abs(F12 - (F1 - 0.5 * F2)).max() <= 1e-11 * np.abs(F1).max()
    b12, b21 = float(np.dot(D1, F2)), float(np.dot(D2, F1))
    assert abs(b12 - b21) <= 1e-11 * abs(b12)
