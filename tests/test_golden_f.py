"""The reference's f-shell known answer (H2O / cc-pVTZ: s, p, d and one f
shell; 65 functions, 2145 packed Fock values at tol 1e-10, identity density,
screening off), kept as a fixture.  Pinned here: the fixture is consistent
with its basis, and the host half of setup plans the f classes for it (the
value checks are in tests/test_oracle_f.py and tests/test_gpu_f.py)."""
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


def test_setup_bytes_plan_the_f_classes():
    # host-only dry run of setup: the f pair classes and the 34 f class plans
    d = load_kat("h2o_ccpvtz")
    full = liberi.setup_bytes(d, 5e-11)
    e = dict(d)
    e["ang_mom"] = [l if l != 4 else 3 for l in d["ang_mom"]]  # the f shell as a d shell
    e["coef_d"] = d["coef_d"] + d["coef_f"]
    e["num_bas"] = d["num_bas"] - 4
    e["atom_loc"] = [a if a <= 26 else a - 4 for a in d["atom_loc"]]
    assert full > liberi.setup_bytes(e, 5e-11) > 0
