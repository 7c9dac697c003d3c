"""The reference's known-answer program driven through the MDI command set
(the order GAMESS sends, liberi_mdi_api.F90:282-420), launches that keep the
state, and the rank split with the shim's reduction of partial F."""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from conftest import load_kat

pytestmark = pytest.mark.gpu


def _send_basis(m, d, coef_f=True):
    m.send(">TYPSCF", "RHF")
    m.send(">NATOMS", d["natoms"])
    m.send(">NUM_BAS", d["num_bas"])
    m.send(">NSH", d["nsh"])
    m.send(">mxgtot", d["mxgtot"])
    for cmd, key in ((">ANGM", "ang_mom"), (">CONTR", "contr_num"), (">SHLLOC", "sh_loc"), (">ATMNUM", "atom_num"),
                     (">ATMLOC", "atom_loc"), (">SBAS", "start_bas"), (">EBAS", "end_bas"), (">EXPON", "exponents"),
                     (">CONTR_COEF_S", "coef_s"), (">CONTR_COEF_P", "coef_p"), (">CONTR_COEF_D", "coef_d"),
                     (">CONTR_COEF_F", "coef_f"), (">COORDS", "coords")):
        m.send(cmd, d[key])
    m.send(">SCHWZ_INT", d["schwrz"])


def test_kat_through_mdi_commands():
    d = load_kat("h2o_ccpvdz")
    m = liberi.MDIEngine()
    _send_basis(m, d)
    for it in range(2):  # one plugin launch per SCF iteration, state kept
        m.send(">AO_DENS", d["density"])
        fa = m.recv("<FOCK")
        assert np.abs(fa - d["fa_ref"]).max() <= d["tol"], it
        m.command("EXIT")
        assert m.terminated
    m.command("EXIT_CONVERGED")  # releases the handle
    with pytest.raises(liberi.LiberiError):
        m.recv("<FOCK")
    m.destroy()


def test_ranks_partials_reduce_to_full_fock():
    d = load_kat("h2o_ccpvdz")
    full = None
    parts = []
    for rank in range(2):
        m = liberi.MDIEngine(rank=rank, nprocs=2)
        _send_basis(m, d)
        m.send(">AO_DENS", d["density"])
        parts.append(m.recv("<FOCK"))
        m.destroy()
    m = liberi.MDIEngine()
    _send_basis(m, d)
    m.send(">AO_DENS", d["density"])
    full = m.recv("<FOCK")
    m.destroy()
    assert np.abs(parts[0] + parts[1] - full).max() <= 1e-12
    assert np.abs(full - d["fa_ref"]).max() <= d["tol"]


def test_nccl_sum_of_partials_single_rank():
    # the library's NCCL reduction of the partial F (one rank on one GPU: the
    # plumbing; more ranks need more GPUs than one call has), inside '<FOCK'
    d = load_kat("h2o_ccpvdz")
    comm = liberi.Comm(liberi.Comm.unique_id(), 0, 1, 0)
    x = np.arange(10, dtype=np.float64)
    assert np.array_equal(comm.reduce_host(x), x)
    m = liberi.MDIEngine()
    m.set_comm(comm)
    _send_basis(m, d)
    m.send(">AO_DENS", d["density"])
    fa = m.recv("<FOCK")
    assert np.abs(fa - d["fa_ref"]).max() <= 1e-10
    m.set_comm(None)
    m.command("EXIT_CONVERGED")
    m.destroy()
    comm.destroy()
