"""Open-shell (UHF) Fock builds on the GPU against the oracle.

F_alpha = J(Da + Db) - K(2 Da), F_beta = J(Da + Db) - K(2 Db) in the units of
the closed-shell build (libERI builds closed-shell F only; its MDI plugin
registers '>AO_DENS_B' / '<FOCK_B' without a beta build,
liberi_mdi_api.F90:395-421).  Tolerances as for the closed-shell path:
max|dF| <= 1e-10 in FP64, |dE| <= 1e-6 Eh in mixed precision."""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from oracle import oracle
from test_gpu_mdi import _send_basis

pytestmark = pytest.mark.gpu


def _spin_densities(n, na, nb, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, max(na, nb))))
    return M.pack(q[:, :na] @ q[:, :na].T), M.pack(q[:, :nb] @ q[:, :nb].T)


def _mol(name):
    b = {"ethane": M.ethane, "random_9": lambda: M.random_molecule(9, seed=11)}[name]()
    b["schwrz"] = oracle.schwarz(b)
    return b


@pytest.mark.parametrize("mol", ["ethane", "random_9"])
def test_uhf_matches_oracle(mol):
    b = _mol(mol)
    n = b["num_bas"]
    Da, Db = _spin_densities(n, 5, 4, seed=3)
    Foa, Fob = oracle.fock_build_uhf(b, Da, Db, schwarz_cut=1e-10)
    h = liberi.liberi_create()
    h.set_option("schwarz_cut", 1e-10)
    liberi.setup_from_basis(h, b)
    Fa, Fb = liberi.fock_uhf(h, Da, Db)
    assert np.abs(Fa - Foa).max() <= 1e-10
    assert np.abs(Fb - Fob).max() <= 1e-10
    # mixed precision
    h.set_option("precision", 1)
    h.set_option("fp32_cut", 1e-7)
    Ma, Mb = liberi.fock_uhf(h, Da, Db)
    w = np.full(Da.size, 2.0)
    w[np.arange(1, n + 1) * np.arange(2, n + 2) // 2 - 1] = 1.0
    for F, Fo, D in ((Ma, Foa, Da), (Mb, Fob, Db)):
        assert 0.5 * abs(np.sum(w * D * (F - Fo))) <= 1e-6
    liberi.liberi_destroy(h)


def test_uhf_closed_shell_limit():
    b = _mol("ethane")
    D = M.density(b["num_bas"], 9, seed=4)
    h = liberi.liberi_create()
    h.set_option("schwarz_cut", 1e-10)
    liberi.setup_from_basis(h, b)
    F = liberi.fock(h, D)
    Fa, Fb = liberi.fock_uhf(h, 0.5 * D, 0.5 * D)
    assert np.abs(Fa - F).max() <= 1e-12 and np.abs(Fb - F).max() <= 1e-12
    # closed-shell builds after an open-shell one are unchanged
    assert np.abs(liberi.fock(h, D) - F).max() <= 1e-12
    liberi.liberi_destroy(h)


def test_mdi_open_shell_commands():
    b = _mol("ethane")
    n = b["num_bas"]
    Da, Db = _spin_densities(n, 5, 4, seed=8)
    Foa, Fob = oracle.fock_build_uhf(b, Da, Db, schwarz_cut=5e-11)
    m = liberi.MDIEngine()
    _send_basis(m, b)
    m.send(">AO_DENS", Da)
    m.send(">AO_DENS_B", Db)
    Fa = m.recv("<FOCK")
    Fb = m.recv("<FOCK_B")
    assert np.abs(Fa - Foa).max() <= 1e-10 and np.abs(Fb - Fob).max() <= 1e-10
    m.command("EXIT_CONVERGED")
    m.destroy()
