"""Algorithmic FP64 operation counts of the engine's quartet kernels.

The roofline numerator of a class kernel is
    FLOPs = N_prim * c_prim(class) + N_shell * c_shell(class)
where N_prim / N_shell are the exact primitive / shell quartet counts of the
plan (liberi_c_get_stats) and the per-unit costs below count the arithmetic
the algorithm needs (add, mul and FMA as 2, one op each for sqrt and
division), mirroring the loop structure of csrc/quartet.cuh:
  per primitive quartet: pair geometry and T, Rys roots and weights
  (2n polynomials of degree 7), per root the recurrence coefficients, the
  2D vertical recurrence, the horizontal transfer on both sides and the
  assembly of the Cartesian block (two multiplies and one add per integral);
  per shell quartet: DIRFCK digestion, 6 multiply-adds per integral plus the
  normalisation and the cut test.
"""


def ncart(l):
    return (l + 1) * (l + 2) // 2


def class_costs(la, lb, lc, ld):
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
    c_prim, c_shell = class_costs(*CLASS_L[k])
    return n_prim * c_prim + n_shell * c_shell


def build_flops(stats):
    return sum(class_flops(k, int(stats["prim_quartets"][k]), int(stats["quartets"][k])) for k in range(21))
