"""MDI plugin command set on the CPU (no device work): payload sizes follow
the state the driver has sent (liberi_mdi_api.F90:282-354), errors as the
C ABI states them."""
import os

import numpy as np
import pytest

from gms_liberi_b200 import liberi
from conftest import ROOT


def test_payloads_follow_the_state():
    m = liberi.MDIEngine()
    assert m.payload(">NSH") == (1, 1)
    assert m.payload(">TYPSCF") == (3, 10)
    m.send(">NATOMS", 3)
    m.send(">NSH", 5)
    m.send(">mxgtot", 4)
    m.send(">NUM_BAS", 7)
    assert m.payload(">ANGM") == (1, 5)
    assert m.payload(">EXPON") == (2, 20)
    assert m.payload(">CONTR_COEF_D") == (2, 20)
    assert m.payload(">COORDS") == (2, 9)
    assert m.payload(">SCHWZ_INT") == (2, 15)
    assert m.payload(">AO_DENS") == (2, 28)
    assert m.payload("<FOCK") == (2, 28)
    assert m.payload("EXIT") == (0, 0)
    assert m.payload(">NSH   ") == (1, 1)  # trailing blanks, as MDI pads commands
    m.destroy()


def test_errors():
    m = liberi.MDIEngine()
    m.send(">NUM_BAS", 7)
    for cmd, code in (("<COORDS", -1), (">FOCK", -1), ("NOPE", -1)):
        with pytest.raises(liberi.LiberiError) as e:
            m.command(cmd)
        assert e.value.code == code
    with pytest.raises(liberi.LiberiError) as e:  # before >SCHWZ_INT
        m.recv("<FOCK")
    assert e.value.code == -2
    with pytest.raises(liberi.LiberiError) as e:  # no open-shell <FOCK yet
        m.recv("<FOCK_B")
    assert e.value.code == -2
    with pytest.raises(liberi.LiberiError) as e:  # wrong payload length
        m._run(">AO_DENS", np.zeros(3), 3)
    assert e.value.code == -3
    with pytest.raises(liberi.LiberiError):
        m.send(">RANK_ID", 2)  # rank 2 of 1
    m.command("EXIT")
    assert m.terminated
    m.destroy()
    with pytest.raises(liberi.LiberiError):
        liberi.MDIEngine(rank=1, nprocs=1)


def test_plugin_shim_compiles_against_mdi_and_mpi_declarations():
    # MDI and MPI are not installed here: the shim is compiled (not linked)
    # against minimal stub declarations of the calls it makes, so its types,
    # signatures and use of the C ABI are checked
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = os.path.join(ROOT, "gms_liberi_b200", "mdi", "liberi_mdi_plugin.c")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "tests", "stubs"),
                        "-I", os.path.join(ROOT, "include"), src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
