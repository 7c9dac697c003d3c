"""The roofline numerator: the per-class operation counts of the reference
algorithm frozen in gms_liberi_b200/flop_constants.json come from the
oracle's op-counting build, which runs the same code as the oracle itself."""
import json
import os

import numpy as np

from gms_liberi_b200 import flops
from gms_liberi_b200 import molecules as M
from oracle import oracle
from conftest import ROOT


def test_constants_cover_every_class():
    with open(os.path.join(ROOT, "gms_liberi_b200", "flop_constants.json")) as f:
        d = json.load(f)
    assert set(d["classes"]) == set(flops.KERNELS)
    for name, v in d["classes"].items():
        assert v["c_prim"] > 0 and v["c_shell"] > 0, name
    c = flops.reference_constants()
    # more angular momentum, more work per primitive quartet
    assert c["int0000"][0] < c["int0111"][0] < c["int1111"][0] < c["int2222"][0]


def test_counting_build_runs_the_oracle_arithmetic():
    b = M.ethane()
    b["schwrz"] = oracle.schwarz(b)
    D = M.density(b["num_bas"], 9, seed=3)
    ops = oracle.count_ops(b, D, schwarz_cut=1e-10)
    _, cnt = oracle.fock_build(b, D, schwarz_cut=1e-10, return_counts=True)
    # the same quartets and primitive quartets as the oracle proper
    assert (ops[:, 2] == cnt[:, 1]).all() and (ops[:, 3] == cnt[:, 3]).all()
    run = ops[:, 2] > 0
    assert (ops[run, 0] > 0).all() and (ops[run, 1] > 0).all()
    # deterministic
    assert (oracle.count_ops(b, D, schwarz_cut=1e-10) == ops).all()


def test_class_flops_formula():
    c_prim, c_shell = flops.reference_constants()["int0101"]
    assert flops.class_flops(4, 1000, 10) == 1000 * c_prim + 10 * c_shell
    assert flops.engine_class_flops(4, 1000, 10) > 0
