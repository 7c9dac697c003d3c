"""Seeded synthetic molecules, bases and densities for the Fock-build workloads.

No public data set is involved: every input is generated here from a seed.
The arrays follow the reference's liberi_setup layout
(src/interface/liberi_interface.F90:72-200): 1-based sh_loc / atom_num /
atom_loc, ang_mom 1=s 2=p 3=d 4=f, per-primitive contraction coefficients that
already contain the GAMESS primitive norms, sp shells split into an s and a p
shell that share exponents, Cartesian d (xx,yy,zz,xy,xz,yz) and f (xxx,yyy,zzz,
xxy,xxz,xyy,yyz,xzz,yzz,xyz), normalised on the axial component.

Workloads:
  * ``h2o_like()``       bent triatomic, STO-3G-shaped, 7 functions.
  * ``ethane()``         staggered C2H6, 6-31G(d)-shaped, 42 functions.
  * ``c60()``            truncated icosahedron, 6-31G(d)-shaped, 900 functions.
  * ``random_molecule()`` C/N/O/H clusters for the batched and serving loops.
  * ``f_triatomic()``    O/C/H with s, p, d and f shells, 38 functions (f checks).
  * ``f_cluster()``      C/N/O/H clusters with f shells on the heavy atoms.
"""
import math

import numpy as np

_ELEM_Z = {"H": 1, "C": 6, "N": 7, "O": 8}

# shell recipes: (kind, K) with kind in "s", "sp", "d"
_SHAPE_631GD_HEAVY = [("s", 6), ("sp", 3), ("sp", 1), ("d", 1)]
_SHAPE_631GD_H = [("s", 3), ("s", 1)]
_SHAPE_STO3G_HEAVY = [("s", 3), ("sp", 3)]
_SHAPE_STO3G_H = [("s", 3)]
# f-bearing shapes: a polarised heavy-atom set with one d and one f
# polarisation shell, H with a p; polarisation exponents ("dpol", "fpol",
# "ppol") in the range of correlation-consistent sets, [0.3, 3]
_SHAPE_F_HEAVY = [("s", 6), ("sp", 3), ("sp", 1), ("dpol", 1), ("fpol", 1)]
_SHAPE_F_H = [("s", 3), ("s", 1), ("ppol", 1)]
_POL_RANGE = (0.3, 3.0)


def _prim_norm(l, a):
    base = (2.0 * a / math.pi) ** 0.75
    if l == 0:
        return base
    if l == 1:
        return 2.0 * math.sqrt(a) * base
    if l == 2:
        # d normalised on the xx component; xy/xz/yz carry the extra sqrt(3)
        return 4.0 * a / math.sqrt(3.0) * base
    # f normalised on xxx: (4a)^(3/2) / sqrt(5!!); the mixed components carry sqrt5 / sqrt15
    return 8.0 * a ** 1.5 / math.sqrt(15.0) * base


def _self_overlap(l, exps, coefs):
    s = 0.0
    for ai, ci in zip(exps, coefs):
        for aj, cj in zip(exps, coefs):
            p = ai + aj
            f = (math.pi / p) ** 1.5
            if l == 1:
                f *= 0.5 / p
            elif l == 2:
                f *= 0.75 / (p * p)
            elif l == 3:
                f *= 1.875 / (p * p * p)
            s += ci * cj * f
    return s


def _contracted(l, exps, raw):
    c = [r * _prim_norm(l, a) for r, a in zip(raw, exps)]
    s = _self_overlap(l, exps, c)
    return [x / math.sqrt(s) for x in c]


def element_basis(elem, shape, lo, hi, seed=0):
    """Per-element list of shells [(l, exps, coefs)], seeded by (seed, Z)."""
    rng = np.random.default_rng([seed, _ELEM_Z[elem]])
    shells = []
    for kind, K in shape:
        elo, ehi = _POL_RANGE if kind.endswith("pol") else (lo, hi)
        kind = kind[0] if kind.endswith("pol") else kind
        exps = np.sort(np.exp(rng.uniform(math.log(elo), math.log(ehi), K)))[::-1].tolist()
        if kind == "s":
            shells.append((0, exps, _contracted(0, exps, rng.uniform(0.1, 1.0, K).tolist())))
        elif kind == "sp":
            shells.append((0, exps, _contracted(0, exps, rng.uniform(0.1, 1.0, K).tolist())))
            shells.append((1, exps, _contracted(1, exps, rng.uniform(0.1, 1.0, K).tolist())))
        elif kind == "p":
            shells.append((1, exps, _contracted(1, exps, rng.uniform(0.1, 1.0, K).tolist())))
        elif kind == "d":
            shells.append((2, exps, _contracted(2, exps, rng.uniform(0.1, 1.0, K).tolist())))
        elif kind == "f":
            shells.append((3, exps, _contracted(3, exps, rng.uniform(0.1, 1.0, K).tolist())))
    return shells


def build_basis(symbols, coords, shells_of):
    """Assemble liberi_setup arrays for atoms ``symbols`` at ``coords`` (bohr)."""
    ang, cnum, shloc, anum, aloc, sbas, ebas = [], [], [], [], [], [], []
    per_shell = []
    bf = 1
    for ia, sym in enumerate(symbols):
        for (l, exps, coefs) in shells_of(sym):
            per_shell.append((l, exps, coefs))
            ang.append(l + 1)
            cnum.append(len(exps))
            anum.append(ia + 1)
            aloc.append(bf)
            sbas.append(bf)
            nc = (1, 3, 6, 10)[l]
            ebas.append(bf + nc - 1)
            bf += nc
    nsh = len(per_shell)
    mx = max(cnum)
    exps_a = np.zeros(mx * nsh)
    cs, cp, cd, cf = (np.zeros(mx * nsh) for _ in range(4))
    for s, (l, exps, coefs) in enumerate(per_shell):
        loc = s * mx
        shloc.append(loc + 1)
        exps_a[loc:loc + len(exps)] = exps
        (cs, cp, cd, cf)[l][loc:loc + len(exps)] = coefs
    nbf = bf - 1
    return {
        "nsh": nsh, "natoms": len(symbols), "num_bas": nbf, "mxgtot": mx,
        "ang_mom": ang, "contr_num": cnum, "sh_loc": shloc, "atom_num": anum,
        "atom_loc": aloc, "start_bas": sbas, "end_bas": ebas,
        "exponents": exps_a, "coef_s": cs, "coef_p": cp, "coef_d": cd,
        "coef_f": cf,
        "coords": np.asarray(coords, dtype=np.float64).reshape(-1),
        "symbols": list(symbols),
    }


def density(nbf, nocc, seed=0):
    """Packed lower triangle of D = 2 C C^T, C orthonormal nbf x nocc."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((nbf, nocc)))
    d = 2.0 * q @ q.T
    return pack(d)


def pack(m):
    n = m.shape[0]
    i, j = np.tril_indices(n)
    # packed index ia(i)+j with ia(i) = i(i-1)/2 (1-based) == row-major lower
    order = np.argsort(i * (i + 1) // 2 + j, kind="stable")
    return np.ascontiguousarray(m[i[order], j[order]])


def unpack(v, n):
    m = np.zeros((n, n))
    i, j = np.tril_indices(n)
    m[i, j] = v[i * (i + 1) // 2 + j]
    m[j, i] = m[i, j]
    return m


def h2o_like(seed=0):
    """Bent triatomic: O at the origin, H at (+-1.430, 1.107, 0) bohr; every
    shell 3 primitives, exponents log-uniform in [0.1, 130]; 7 functions."""
    sym = ["O", "H", "H"]
    xyz = [[0.0, 0.0, 0.0], [1.430, 1.107, 0.0], [-1.430, 1.107, 0.0]]
    heavy = element_basis("O", _SHAPE_STO3G_HEAVY, 0.1, 130.0, seed)
    hyd = element_basis("H", _SHAPE_STO3G_H, 0.1, 130.0, seed)
    return build_basis(sym, xyz, lambda s: heavy if s != "H" else hyd)


def _basis_631gd(seed=0):
    cache = {}

    def shells_of(sym):
        if sym not in cache:
            shape = _SHAPE_631GD_H if sym == "H" else _SHAPE_631GD_HEAVY
            cache[sym] = element_basis(sym, shape, 0.1, 3000.0, seed)
        return cache[sym]

    return shells_of


def ethane(seed=0):
    """Staggered C2H6: C-C 2.91 bohr, C-H 2.06 bohr, tetrahedral angles."""
    cc, ch = 2.91, 2.06
    th = math.radians(180.0 - 109.4712206)
    sym, xyz = ["C", "C"], [[0, 0, cc / 2], [0, 0, -cc / 2]]
    for k in range(3):
        ph = math.radians(120.0 * k)
        sym.append("H")
        xyz.append([ch * math.sin(th) * math.cos(ph), ch * math.sin(th) * math.sin(ph),
                    cc / 2 + ch * math.cos(th)])
    for k in range(3):
        ph = math.radians(60.0 + 120.0 * k)
        sym.append("H")
        xyz.append([ch * math.sin(th) * math.cos(ph), ch * math.sin(th) * math.sin(ph),
                    -cc / 2 - ch * math.cos(th)])
    return build_basis(sym, xyz, _basis_631gd(seed))


def c60_coords(b66=2.65, b56=2.74):
    """Truncated icosahedron: every icosahedron edge A->B gives the vertex
    A + t(B - A).  Pentagon (5:6) bonds have length t*e and hexagon-hexagon
    (6:6) bonds (1 - 2t)*e, which fixes t and the icosahedron edge e."""
    t = b56 / (b56 * 2.0 + b66)
    e = b56 / t
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    ico = []
    for a in (-1.0, 1.0):
        for b in (-phi, phi):
            ico += [(0.0, a, b), (a, b, 0.0), (b, 0.0, a)]
    ico = np.array(ico) * (e / 2.0)
    verts = []
    for i in range(12):
        for j in range(12):
            if i != j and abs(np.linalg.norm(ico[i] - ico[j]) - e) < 1e-6:
                verts.append(ico[i] + t * (ico[j] - ico[i]))
    verts = np.array(verts)
    assert verts.shape == (60, 3)
    return verts


def c60(seed=0):
    xyz = c60_coords()
    return build_basis(["C"] * 60, xyz, _basis_631gd(seed))


def random_molecule(natoms, seed, rho=0.01, dmin=1.9):
    """C/N/O/H in 3:1:1:5 proportions, positions rejection-sampled with a
    minimum separation of ``dmin`` bohr inside a sphere at ``rho`` atoms/bohr^3."""
    rng = np.random.default_rng([seed, natoms, 7919])
    pool = ["C"] * 3 + ["N"] + ["O"] + ["H"] * 5
    sym = [pool[i] for i in rng.integers(0, len(pool), natoms)]
    if all(s == "H" for s in sym):
        sym[0] = "C"
    R = (3.0 * natoms / (4.0 * math.pi * rho)) ** (1.0 / 3.0)
    pts = []
    tries = 0
    while len(pts) < natoms:
        tries += 1
        v = rng.uniform(-R, R, 3)
        if np.dot(v, v) > R * R:
            continue
        if all(np.linalg.norm(v - p) >= dmin for p in pts):
            pts.append(v)
        if tries > 1000000:
            raise RuntimeError("rejection sampling failed")
    return build_basis(sym, np.array(pts), _basis_631gd(0))


def nocc_of(basis):
    """Closed-shell occupation from nuclear charges (neutral molecule)."""
    z = sum(_ELEM_Z[s] for s in basis["symbols"])
    return z // 2


def _basis_f(seed=0):
    def shells_of(sym):
        if sym == "H":
            return element_basis("H", _SHAPE_F_H, 0.12, 20.0, seed)
        return element_basis(sym, _SHAPE_F_HEAVY, 0.15, 3000.0, seed)
    return shells_of


def f_triatomic(seed=0):
    """Three atoms with s, p, d and f shells (38 functions): O with s(3), s(1),
    p(1), d(1), f(1); C with s(1), s(2), p(2), f(1); H with s(2), s(1)."""
    shapes = {"O": [("s", 3), ("sp", 1), ("d", 1), ("f", 1)],
              "C": [("s", 1), ("sp", 2), ("f", 1)],
              "H": [("s", 2), ("s", 1)]}

    def shells_of(sym):
        return element_basis(sym, shapes[sym], 0.2, 40.0, seed)

    xyz = np.array([[0.0, 0.0, 0.0], [0.4, 2.1, 1.3], [-1.7, -0.6, 1.1]])
    return build_basis(["O", "C", "H"], xyz, shells_of)


def f_cluster(natoms, seed=0, rho=0.01, dmin=1.9):
    """C/N/O/H cluster (as random_molecule) with an f shell and a d shell on
    every heavy atom and a p shell on every H."""
    b = random_molecule(natoms, seed, rho, dmin)
    xyz = np.asarray(b["coords"]).reshape(-1, 3)
    return build_basis(b["symbols"], xyz, _basis_f(seed))
