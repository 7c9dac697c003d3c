#!/usr/bin/env python
"""Freeze the per-class operation counts of the reference algorithm for the
roofline numerator: FLOPs(class) = N_prim * c_prim + N_shell * c_shell.

The counts come from the oracle's op-counting build (oracle/opcount.cpp:
the oracle's restatement of the reference algorithm -- Boys-moment Rys rules
for the rotated-axis classes, RYSDS + RYSGW for the Rys classes, recurrences,
assembly and DIRFCK -- compiled with a scalar type that counts add,
subtract, multiply, divide, exp, sqrt, acos and cos as one operation each)
run on the C60 6-31G(d)-shaped benchmark workload (Schwarz cut 1e-10) over a
hashed 1/SAMPLE sample of every class's screened quartets:
    c_prim  = operations in primitive-quartet work / primitive quartets,
    c_shell = operations in shell-quartet work (component normalisation and
              DIRFCK digestion) / shell quartets.
TEST INFRASTRUCTURE: this script runs the oracle; its output, the JSON file
gms_liberi_b200/flop_constants.json, is plain data that flops.py reads.

    python oracle/make_flop_constants.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[0] = ROOT  # the package root, not this folder (oracle.py would shadow the package)

import numpy as np  # noqa: E402

from gms_liberi_b200 import molecules as M  # noqa: E402
from oracle import oracle  # noqa: E402

SAMPLE = 20
OUT = os.path.join(ROOT, "gms_liberi_b200", "flop_constants.json")


def main():
    b = M.c60()
    b["schwrz"] = oracle.schwarz(b)
    D = M.density(b["num_bas"], 180, seed=0)
    t0 = time.time()
    c = oracle.count_ops(b, D, schwarz_cut=1e-10, sample_mod=SAMPLE)
    secs = time.time() - t0
    classes = {}
    for k in range(21):
        if c[k, 2] <= 0 or c[k, 3] <= 0:
            continue
        classes[oracle.KERNELS[k]] = {"c_prim": round(float(c[k, 0] / c[k, 2]), 3),
                                      "c_shell": round(float(c[k, 1] / c[k, 3]), 3),
                                      "prim_quartets_counted": int(c[k, 2]),
                                      "shell_quartets_counted": int(c[k, 3])}
    out = {"source": "oracle op-counting build (oracle/opcount.cpp) of the restated reference algorithm",
           "workload": "C60 truncated icosahedron, 6-31G(d)-shaped basis, D = 2CC^T (180 columns, seed 0), "
                       "Schwarz cut 1e-10, hashed 1/%d sample of each class's screened quartets" % SAMPLE,
           "operations": "add, subtract, multiply, divide, exp, sqrt, acos, cos: one each; no fused multiply-add",
           "classes": classes}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print("wrote %s (%d classes, %.1f s)" % (OUT, len(classes), secs))


if __name__ == "__main__":
    main()
