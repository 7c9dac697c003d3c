"""Independent two-electron integrals for the oracle's f-shell checks.

TEST INFRASTRUCTURE: a second, unrelated evaluation of (ab|cd) over Cartesian
Gaussians, used to check the oracle's Rys-quadrature restatement where the
reference ships no usable known answer (f shells).  Method: McMurchie-Davidson
(L. E. McMurchie and E. R. Davidson, J. Comput. Phys. 26 (1978) 218) -- each
product of two Gaussians expanded in Hermite Gaussians (coefficients E^{ij}_t
by the two-term recurrences), the Coulomb interaction of two Hermite Gaussians
from the auxiliary integrals R^n_{tuv} (Boys functions from scipy's regularised
incomplete gamma), the four-centre integral a double contraction
sum_{tuv} E^{ab}_{tuv} sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd} R_{t+tau,...}.
Component order and normalisation are derived here from first principles:
GAMESS order within each shell, each Cartesian component normalised, i.e. the
input coefficient (normalised for x^l) times sqrt((2l-1)!! / ((2lx-1)!!
(2ly-1)!! (2lz-1)!!)).  The Fock matrix follows from the integrals by the
DIRFCK updates over unique function quadruples.  Pure numpy; small molecules
only.
"""
import math

import numpy as np
from scipy.special import gamma, gammainc

COMP = {0: [(0, 0, 0)], 1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
        2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
        3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2),
            (0, 1, 2), (1, 1, 1)]}


def _dfact(n):
    return 1 if n <= 0 else n * _dfact(n - 2)


def _comp_norm(l, lx, ly, lz):
    return math.sqrt(_dfact(2 * l - 1) / (_dfact(2 * lx - 1) * _dfact(2 * ly - 1) * _dfact(2 * lz - 1)))


def _boys(nmax, T):
    m = np.arange(nmax + 1)
    if T < 1e-12:
        return 1.0 / (2 * m + 1)
    return gamma(m + 0.5) * gammainc(m + 0.5, T) / (2 * T ** (m + 0.5))


def _hermite_1d(la, lb, a, b, xab):
    """E[i, j, t] for one Cartesian direction, xab = A - B."""
    p = a + b
    xpa, xpb = -b / p * xab, a / p * xab
    E = np.zeros((la + 1, lb + 1, la + lb + 2))
    E[0, 0, 0] = math.exp(-a * b / p * xab * xab)
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            src, x = ((i - 1, j), xpa) if i > 0 else ((i, j - 1), xpb)
            for t in range(i + j + 1):
                v = x * E[src + (t,)] + (t + 1) * E[src + (t + 1,)]
                if t > 0:
                    v += E[src + (t - 1,)] / (2 * p)
                E[i, j, t] = v
    return E


def _aux(L, alpha, pq):
    """R_{tuv} = R^0_{tuv}(alpha, PQ) for t + u + v <= L."""
    F = _boys(L, alpha * float(pq.dot(pq)))
    R = np.zeros((L + 1, L + 2, L + 2, L + 2))
    for n in range(L + 1):
        R[n, 0, 0, 0] = (-2 * alpha) ** n * F[n]
    X, Y, Z = pq
    for tot in range(1, L + 1):
        for n in range(L - tot + 1):
            for t in range(tot + 1):
                for u in range(tot - t + 1):
                    v = tot - t - u
                    if t > 0:
                        r = X * R[n + 1, t - 1, u, v] + ((t - 1) * R[n + 1, t - 2, u, v] if t > 1 else 0.0)
                    elif u > 0:
                        r = Y * R[n + 1, t, u - 1, v] + ((u - 1) * R[n + 1, t, u - 2, v] if u > 1 else 0.0)
                    else:
                        r = Z * R[n + 1, t, u, v - 1] + ((v - 1) * R[n + 1, t, u, v - 2] if v > 1 else 0.0)
                    R[n, t, u, v] = r
    return R[0]


def _pair_matrix(la, lb, a, b, ab, ket):
    """Hermite coefficients of every component pair: rows (i, j), columns (t, u, v) dense."""
    E = [_hermite_1d(la, lb, a, b, ab[x]) for x in range(3)]
    L = la + lb + 1
    sign = (-1.0) ** np.arange(L) if ket else np.ones(L)
    rows = []
    for ax, ay, az in COMP[la]:
        for bx, by, bz in COMP[lb]:
            ex = E[0][ax, bx, :L] * sign
            ey = E[1][ay, by, :L] * sign
            ez = E[2][az, bz, :L] * sign
            rows.append(np.einsum("t,u,v->tuv", ex, ey, ez).ravel())
    return np.array(rows)


def shells_of(basis):
    out = []
    for s in range(int(basis["nsh"])):
        l = int(basis["ang_mom"][s]) - 1
        lo = int(basis["sh_loc"][s]) - 1
        k = int(basis["contr_num"][s])
        coef = [basis["coef_s"], basis["coef_p"], basis["coef_d"], basis["coef_f"]][l]
        at = int(basis["atom_num"][s]) - 1
        out.append(dict(l=l, a=np.asarray(basis["exponents"][lo:lo + k], dtype=float),
                        c=np.asarray(coef[lo:lo + k], dtype=float),
                        R=np.asarray(basis["coords"][3 * at:3 * at + 3], dtype=float),
                        f0=int(basis["atom_loc"][s]) - 1))
    return out


def shell_quartet(A, B, C, D):
    """Contracted, normalised (AB|CD) block [na, nb, nc, nd]."""
    la, lb, lc, ld = A["l"], B["l"], C["l"], D["l"]
    L1, L2 = la + lb + 1, lc + ld + 1
    t1, t2 = np.arange(L1), np.arange(L2)
    it = t1[:, None, None, None, None, None] + t2[None, None, None, :, None, None]
    iu = t1[None, :, None, None, None, None] + t2[None, None, None, None, :, None]
    iv = t1[None, None, :, None, None, None] + t2[None, None, None, None, None, :]
    out = np.zeros((len(COMP[la]) * len(COMP[lb]), len(COMP[lc]) * len(COMP[ld])))
    ab, cd = A["R"] - B["R"], C["R"] - D["R"]
    for a, ca in zip(A["a"], A["c"]):
        for b, cb in zip(B["a"], B["c"]):
            p = a + b
            P = (a * A["R"] + b * B["R"]) / p
            Hab = _pair_matrix(la, lb, a, b, ab, False)
            for c, cc in zip(C["a"], C["c"]):
                for d, cdd in zip(D["a"], D["c"]):
                    q = c + d
                    Q = (c * C["R"] + d * D["R"]) / q
                    Hcd = _pair_matrix(lc, ld, c, d, cd, True)
                    R = _aux(la + lb + lc + ld, p * q / (p + q), P - Q)
                    M = R[it, iu, iv].reshape(L1 ** 3, L2 ** 3)
                    pre = 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * ca * cb * cc * cdd
                    out += pre * (Hab @ M @ Hcd.T)
    out = out.reshape(len(COMP[la]), len(COMP[lb]), len(COMP[lc]), len(COMP[ld]))
    for axis, l in enumerate((la, lb, lc, ld)):
        shape = [1, 1, 1, 1]
        shape[axis] = -1
        out = out * np.array([_comp_norm(l, *x) for x in COMP[l]]).reshape(shape)
    return out


def eri_tensor(basis):
    """Full (ij|kl) over basis functions, from the unique shell quartets."""
    sh = shells_of(basis)
    n = int(basis["num_bas"])
    G = np.zeros((n, n, n, n))
    pairs = [(i, j) for i in range(len(sh)) for j in range(i + 1)]
    for x, (i, j) in enumerate(pairs):
        for (k, l) in pairs[:x + 1]:
            A, B, C, D = sh[i], sh[j], sh[k], sh[l]
            v = shell_quartet(A, B, C, D)
            sa = slice(A["f0"], A["f0"] + v.shape[0])
            sb = slice(B["f0"], B["f0"] + v.shape[1])
            sc = slice(C["f0"], C["f0"] + v.shape[2])
            sd = slice(D["f0"], D["f0"] + v.shape[3])
            for blk, idx in ((v, (sa, sb, sc, sd)), (v.transpose(1, 0, 2, 3), (sb, sa, sc, sd)),
                             (v.transpose(0, 1, 3, 2), (sa, sb, sd, sc)),
                             (v.transpose(1, 0, 3, 2), (sb, sa, sd, sc))):
                G[idx] = blk
                G[idx[2], idx[3], idx[0], idx[1]] = blk.transpose(2, 3, 0, 1)
    return G


def fock_from_eri(G, density, exchange_density=None):
    """Packed F from the DIRFCK updates (F(ij) += 4 v D(kl), F(ik) -= v X(jl), ...;
    v halved for i = j, k = l and ij = kl) over unique function quadruples; the
    exchange updates read X = exchange_density (default: the same D)."""
    n = G.shape[0]
    tri = np.zeros((n, n), dtype=np.int64)
    for i in range(n):
        for j in range(i + 1):
            tri[i, j] = tri[j, i] = i * (i + 1) // 2 + j
    D = np.asarray(density, dtype=float)
    X = D if exchange_density is None else np.asarray(exchange_density, dtype=float)
    F = np.zeros_like(D)
    iu, ju = np.tril_indices(n)
    for i, j in zip(iu, ju):
        ij = tri[i, j]
        k, l = iu[: ij + 1], ju[: ij + 1]  # pairs kl <= ij
        v = G[i, j, k, l].copy()
        if i == j:
            v *= 0.5
        v[k == l] *= 0.5
        v[-1] *= 0.5  # kl == ij
        kl = tri[k, l]
        F[ij] += 4.0 * np.dot(v, D[kl])
        np.add.at(F, kl, 4.0 * v * D[ij])
        np.add.at(F, tri[i, k], -v * X[tri[j, l]])
        np.add.at(F, tri[j, l], -v * X[tri[i, k]])
        np.add.at(F, tri[i, l], -v * X[tri[j, k]])
        np.add.at(F, tri[j, k], -v * X[tri[i, l]])
    return F
