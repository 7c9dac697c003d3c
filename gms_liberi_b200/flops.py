"""Algorithmic operation counts of the Fock build, the roofline numerator.

For a class kernel
    FLOPs = N_prim * c_prim(class) + N_shell * c_shell(class)
where N_prim / N_shell are the exact primitive / shell quartet counts of the
plan (liberi_c_get_stats).  Two sets of per-unit costs:

  * reference algorithm (the primary figure): c_prim and c_shell frozen in
    flop_constants.json beside this file, counted by the oracle's op-counting
    build on the C60 benchmark workload (oracle/make_flop_constants.py): the
    operations of the restated reference algorithm -- Boys-moment Rys rules
    for the rotated-axis classes, the 35-point Stieltjes procedure and
    Golub-Welsch step per primitive quartet for the Rys classes, recurrences,
    assembly and DIRFCK digestion; one operation each for add, subtract,
    multiply, divide, exp, sqrt, acos and cos.  Redundant work in the engine
    therefore cannot raise this figure.
  * engine count (secondary): the arithmetic of the engine's own loops
    (csrc/quartet.cuh), add, mul and FMA as 2: per primitive quartet the pair
    geometry and T, the Rys roots and weights (2n polynomials of degree 7), per
    root the recurrence coefficients, the 2D vertical recurrence, the
    horizontal transfer and the assembly; per shell quartet the digestion.
"""
import json
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
KERNELS = ["int0000", "int0001", "int0011", "int0111", "int0101", "int1111",
           "int0002", "int0012", "int0102", "int0112", "int0022", "int0122",
           "int1102", "int0202", "int2211", "int2121", "int2120", "int2111",
           "int2220", "int2221", "int2222"]
_REF = None


def reference_constants():
    """{class name: (c_prim, c_shell)} of the reference algorithm."""
    global _REF
    if _REF is None:
        with open(os.path.join(_HERE, "flop_constants.json")) as f:
            d = json.load(f)
        _REF = {k: (v["c_prim"], v["c_shell"]) for k, v in d["classes"].items()}
    return _REF


def ncart(l):
    return (l + 1) * (l + 2) // 2


def engine_costs(la, lb, lc, ld):
    lab, lcd = la + lb, lc + ld
    n = (lab + lcd) // 2 + 1
    nc = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    setup = 20
    roots = 2 * n * 14 + 7
    per_root = 20
    vrr = 0
    for i in range(lab):
        vrr += 1 if i == 0 else 4
    for k in range(lcd):
        for i in range(lab + 1):
            vrr += 1 + (2 if k > 0 else 0) + (2 if i > 0 else 0)
    hrr = 0
    for b in range(1, lb + 1):
        hrr += (lab - b + 1) * (lcd + 1) * 2
    for d in range(1, ld + 1):
        hrr += (la + 1) * (lb + 1) * (lcd - d + 1) * 2
    asm = 3 * nc
    c_prim = setup + roots + n * (per_root + 3 * (vrr + hrr) + asm)
    c_shell = 14 * nc
    return c_prim, c_shell


# engine orientation of the 21 reference classes (driver order)
CLASS_L = [(0, 0, 0, 0), (0, 0, 1, 0), (0, 0, 1, 1), (1, 0, 1, 1), (1, 0, 1, 0), (1, 1, 1, 1),
           (0, 0, 2, 0), (0, 0, 2, 1), (1, 0, 2, 0), (1, 0, 2, 1), (0, 0, 2, 2), (1, 0, 2, 2),
           (1, 1, 2, 0), (2, 0, 2, 0), (2, 2, 1, 1), (2, 1, 2, 1), (2, 1, 2, 0), (2, 1, 1, 1),
           (2, 2, 2, 0), (2, 2, 2, 1), (2, 2, 2, 2)]


def class_flops(k, n_prim, n_shell):
    """Reference-algorithm operations of class k (driver order)."""
    c_prim, c_shell = reference_constants()[KERNELS[k]]
    return n_prim * c_prim + n_shell * c_shell


def engine_class_flops(k, n_prim, n_shell):
    """The engine's own arithmetic for class k."""
    c_prim, c_shell = engine_costs(*CLASS_L[k])
    return n_prim * c_prim + n_shell * c_shell


def build_flops(stats):
    return sum(class_flops(k, int(stats["prim_quartets"][k]), int(stats["quartets"][k])) for k in range(21))


def engine_build_flops(stats):
    return sum(engine_class_flops(k, int(stats["prim_quartets"][k]), int(stats["quartets"][k])) for k in range(21))
