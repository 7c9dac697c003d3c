"""The reference's f-shell known answer (H2O / cc-pVTZ: s, p, d and one f
shell; 65 functions, 2145 packed Fock values at tol 1e-10, identity density,
screening off), kept as a fixture for the f-shell classes, which this engine
does not build yet.  Pinned here: the fixture is consistent, and setup through
the C ABI rejects its f shell cleanly (LIBERI_E_UNSUPPORTED naming the shell)
rather than building a partial F."""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from conftest import load_kat

NCART = {1: 1, 2: 3, 3: 6, 4: 10}


def test_f_fixture_is_consistent():
    d = load_kat("h2o_ccpvtz")
    n, nsh = d["num_bas"], d["nsh"]
    assert (n, nsh, d["natoms"]) == (65, 22, 3)
    assert len(d["fa_ref"]) == n * (n + 1) // 2 == 2145
    assert sum(NCART[l] for l in d["ang_mom"]) == n
    ends = d["atom_loc"][1:] + [n + 1]
    assert all(a + NCART[l] == e for a, l, e in zip(d["atom_loc"], d["ang_mom"], ends))
    f_shells = [i for i, l in enumerate(d["ang_mom"]) if l == 4]
    assert f_shells == [9]
    assert d["coef_f"][d["sh_loc"][9] - 1] > 0
    assert np.isfinite(d["fa_ref"]).all()


def test_setup_rejects_the_f_shell():
    d = load_kat("h2o_ccpvtz")
    h = liberi.liberi_create()
    with pytest.raises(liberi.LiberiError) as e:
        liberi.liberi_setup(h, d["nsh"], d["natoms"], d["num_bas"], d["mxgtot"], d["ang_mom"], d["contr_num"],
                            d["sh_loc"], d["atom_num"], d["atom_loc"], d["start_bas"], d["end_bas"], d["exponents"],
                            d["coef_s"], d["coef_p"], d["coef_d"], d["coef_f"], d["coords"], d["schwrz"], 0, 1)
    assert e.value.code == -6
    assert "shell 10" in str(e.value) and "f shell" in str(e.value)
    liberi.liberi_destroy(h)
