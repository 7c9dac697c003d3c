// quartet.cuh -- sm_100a device code of the quartet classes (included by the
// per-class translation units k_*.cu and by kernels.cu).
//
// One templated kernel per reference quartet class intABCD
// (src/rhf/rot_axis/int*.F90, driver order src/liberi_driver.F90:69-102).
// A thread owns one screened shell quartet (bra pair P, ket pair Q):
//   1. decode the flat work index into (P, Q) from the class plan: bra pairs
//      sorted by Schwarz value, per bra a prefix of the sorted ket list;
//   2. loop over kept primitive pairs (ket outer, bra inner, as the
//      reference does, e.g. int0001.F90:220-287), evaluate Rys roots and
//      weights from the piecewise tables, build 2D integrals with the
//      vertical and horizontal recurrences in registers and contract the
//      Cartesian block;
//   3. digest the block into the packed Fock matrix with the reference's
//      DIRFCK rules (unique components for identical shells, 0.5 factors,
//      skip |v| < cut, six updates; int0000.F90:241-311,
//      int2222_rysgen.F90:11176-11338) using FP64 atomics.
// The FP32 instantiation evaluates steps 2's recurrences and contraction in
// single precision (roots, weights and pair prefactors stay FP64) for the
// quartets whose Schwarz bound falls below the mixed-precision cut; its
// integrals are digested into the same FP64 Fock matrix.
#pragma once
#include <cstdio>

#include "engine.h"

namespace liberi {


// ---- Cartesian components: p = x,y,z ; d = xx,yy,zz,xy,xz,yz ---------------
__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int cxp(int l, int c) {
    return l == 0 ? 0 : (l == 1 ? (c == 0 ? 1 : 0) : (c == 0 ? 2 : ((c == 3 || c == 4) ? 1 : 0)));
}
__host__ __device__ constexpr int cyp(int l, int c) {
    return l == 0 ? 0 : (l == 1 ? (c == 1 ? 1 : 0) : (c == 1 ? 2 : ((c == 3 || c == 5) ? 1 : 0)));
}
__host__ __device__ constexpr int czp(int l, int c) {
    return l == 0 ? 0 : (l == 1 ? (c == 2 ? 1 : 0) : (c == 2 ? 2 : ((c == 4 || c == 5) ? 1 : 0)));
}
// number of sqrt(3) factors (xy, xz, yz of a d shell)
__host__ __device__ constexpr int cs3(int l, int c) { return (l == 2 && c >= 3) ? 1 : 0; }

__device__ __forceinline__ long long tri1(long long i, long long j) {  // 1-based ia(max)+min
    return i >= j ? i * (i - 1) / 2 + j : j * (j - 1) / 2 + i;
}

// ---- Rys roots/weights -------------------------------------------------------
template <int N>
__device__ __forceinline__ void rys_eval(double T, double thr, bool strict,
                                         const double *__restrict__ tab, double *u, double *w) {
    bool asym = strict ? (T > thr) : (T >= thr);
    if (asym) {
        double it = 1.0 / T, sq = sqrt(it);
        const double *hr = tab + rys_herm_off(N);
#pragma unroll
        for (int i = 0; i < N; i++) {
            u[i] = __ldg(hr + i) * it;
            w[i] = __ldg(hr + MAXROOT + i) * sq;
        }
        return;
    }
    int k = (int)T;
    double x = 2.0 * (T - (double)k) - 1.0;
    const double *base = tab + rys_table_off(N) + (size_t)k * (2 * N * RYS_NCOEF);
#pragma unroll
    for (int f = 0; f < 2 * N; f++) {
        const double *c = base + f * RYS_NCOEF;
        double v = __ldg(c + RYS_DEG);
#pragma unroll
        for (int j = RYS_DEG - 1; j >= 0; j--) v = fma(v, x, __ldg(c + j));
        if (f < N) u[f] = v; else w[f - N] = v;
    }
}

// ---- recurrences -------------------------------------------------------------
template <int LAB, int LCD, typename R>
__device__ __forceinline__ void vrr(R (&g)[LAB + 1][LCD + 1], R c00, R cp00, R b10, R b01,
                                    R b00, R g00) {
    g[0][0] = g00;
#pragma unroll
    for (int i = 0; i < LAB; i++) {
        R v = c00 * g[i][0];
        if (i > 0) v += R(i) * b10 * g[i - 1][0];
        g[i + 1][0] = v;
    }
#pragma unroll
    for (int k = 0; k < LCD; k++) {
#pragma unroll
        for (int i = 0; i <= LAB; i++) {
            R v = cp00 * g[i][k];
            if (k > 0) v += R(k) * b01 * g[i][k - 1];
            if (i > 0) v += R(i) * b00 * g[i - 1][k];
            g[i][k + 1] = v;
        }
    }
}

// horizontal transfer: I[a][b][c][d] from g[e][f], e<=LA+LB, f<=LC+LD
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void hrr(const R (&g)[LA + LB + 1][LC + LD + 1], R ab, R cd,
                                    R (&I)[LA + 1][LB + 1][LC + 1][LD + 1]) {
    constexpr int LAB = LA + LB, LCD = LC + LD;
    R h[LAB + 1][LB + 1][LCD + 1];
#pragma unroll
    for (int e = 0; e <= LAB; e++)
#pragma unroll
        for (int f = 0; f <= LCD; f++) h[e][0][f] = g[e][f];
#pragma unroll
    for (int b = 1; b <= LB; b++)
#pragma unroll
        for (int a = 0; a <= LAB - b; a++)
#pragma unroll
            for (int f = 0; f <= LCD; f++) h[a][b][f] = h[a + 1][b - 1][f] + ab * h[a][b - 1][f];
#pragma unroll
    for (int a = 0; a <= LA; a++)
#pragma unroll
        for (int b = 0; b <= LB; b++) {
            R k2[LCD + 1][LD + 1];
#pragma unroll
            for (int f = 0; f <= LCD; f++) k2[f][0] = h[a][b][f];
#pragma unroll
            for (int d = 1; d <= LD; d++)
#pragma unroll
                for (int c = 0; c <= LCD - d; c++) k2[c][d] = k2[c + 1][d - 1] + cd * k2[c][d - 1];
#pragma unroll
            for (int c = 0; c <= LC; c++)
#pragma unroll
                for (int d = 0; d <= LD; d++) I[a][b][c][d] = k2[c][d];
        }
}

// ---- contracted Cartesian block of one shell quartet -------------------------
template <int LA, int LB, int LC, int LD, typename R>
struct Quartet {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NCART = NA * NB * NC * ND;
    static constexpr int LAB = LA + LB, LCD = LC + LD;
    static constexpr int NR = (LAB + LCD) / 2 + 1;

    __device__ __forceinline__ static int64_t eval(const DevBasis &b, int P, int Q, double thr,
                                                    bool strict, const double *__restrict__ tab,
                                                    R (&acc)[NCART]) {
        const int2 sab = b.pair_shell[P], scd = b.pair_shell[Q];
        const double4 A = b.shell_xyz[sab.x], B = b.shell_xyz[sab.y];
        const double4 C = b.shell_xyz[scd.x], D = b.shell_xyz[scd.y];
        const R abx = R(A.x - B.x), aby = R(A.y - B.y), abz = R(A.z - B.z);
        const R cdx = R(C.x - D.x), cdy = R(C.y - D.y), cdz = R(C.z - D.z);
#pragma unroll
        for (int i = 0; i < NCART; i++) acc[i] = R(0);
        const int p0 = b.pair_prim0[P], np = b.pair_nprim[P];
        const int q0 = b.pair_prim0[Q], nq = b.pair_nprim[Q];
        for (int kq = q0; kq < q0 + nq; kq++) {
            const double4 Qp = b.prim_P[kq];
            const double Kq = b.prim_K[kq];
            const double q = Qp.w;
            const double hq = 0.5 / q;
            for (int kp = p0; kp < p0 + np; kp++) {
                const double4 Pp = b.prim_P[kp];
                const double Kp = b.prim_K[kp];
                const double p = Pp.w;
                const double hp = 0.5 / p;
                const double rs = rsqrt(p + q);
                const double ipq = rs * rs;
                const double pqx = Pp.x - Qp.x, pqy = Pp.y - Qp.y, pqz = Pp.z - Qp.z;
                const double rho = p * q * ipq;
                const double T = rho * (pqx * pqx + pqy * pqy + pqz * pqz);
                double u[NR], w[NR];
                rys_eval<NR>(T, thr, strict, tab, u, w);
                const double pref = Kp * Kq * rs;
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const double ui = u[r] * ipq;
                    const double fq = q * ui, fp = p * ui;
                    const R b00 = R(0.5 * ui);
                    const R b10 = R(hp * (1.0 - fq));
                    const R b01 = R(hq * (1.0 - fp));
                    R gx[LAB + 1][LCD + 1], gy[LAB + 1][LCD + 1], gz[LAB + 1][LCD + 1];
                    vrr<LAB, LCD, R>(gx, R((Pp.x - A.x) - fq * pqx), R((Qp.x - C.x) + fp * pqx),
                                     b10, b01, b00, R(1));
                    vrr<LAB, LCD, R>(gy, R((Pp.y - A.y) - fq * pqy), R((Qp.y - C.y) + fp * pqy),
                                     b10, b01, b00, R(1));
                    vrr<LAB, LCD, R>(gz, R((Pp.z - A.z) - fq * pqz), R((Qp.z - C.z) + fp * pqz),
                                     b10, b01, b00, R(w[r] * pref));
                    R ix[LA + 1][LB + 1][LC + 1][LD + 1], iy[LA + 1][LB + 1][LC + 1][LD + 1],
                        iz[LA + 1][LB + 1][LC + 1][LD + 1];
                    hrr<LA, LB, LC, LD, R>(gx, abx, cdx, ix);
                    hrr<LA, LB, LC, LD, R>(gy, aby, cdy, iy);
                    hrr<LA, LB, LC, LD, R>(gz, abz, cdz, iz);
#pragma unroll(NCART > 81 ? 1 : NA)
                    for (int ia = 0; ia < NA; ia++)
#pragma unroll
                        for (int ib = 0; ib < NB; ib++)
#pragma unroll
                            for (int ic = 0; ic < NC; ic++)
#pragma unroll
                                for (int id = 0; id < ND; id++) {
                                    const int n = ((ia * NB + ib) * NC + ic) * ND + id;
                                    acc[n] += ix[cxp(LA, ia)][cxp(LB, ib)][cxp(LC, ic)][cxp(LD, id)] *
                                              iy[cyp(LA, ia)][cyp(LB, ib)][cyp(LC, ic)][cyp(LD, id)] *
                                              iz[czp(LA, ia)][czp(LB, ib)][czp(LC, ic)][czp(LD, id)];
                                }
                }
            }
        }
        return (int64_t)np * nq;
    }
};

// ---- DIRFCK digestion ----------------------------------------------------------
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void digest(const R *acc, int bfA, int bfB, int bfC, int bfD,
                                       bool iandj, bool kandl, bool same, double cut,
                                       const double *__restrict__ Dm, double *F) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr bool can_same = (LA == LC) && (LB == LD);
    const double s3 = 1.7320508075688772935;
#pragma unroll(NA * NB * NC * ND > 81 ? 1 : NA)
    for (int ia = 0; ia < NA; ia++)
#pragma unroll
        for (int ib = 0; ib < NB; ib++) {
            if (LA == LB && iandj && ib > ia) continue;
#pragma unroll
            for (int ic = 0; ic < NC; ic++)
#pragma unroll
                for (int id = 0; id < ND; id++) {
                    if (LC == LD && kandl && id > ic) continue;
                    if (can_same && same) {
                        const int oij = iandj ? ia * (ia + 1) / 2 + ib : ia * NB + ib;
                        const int okl = kandl ? ic * (ic + 1) / 2 + id : ic * ND + id;
                        if (okl > oij) continue;
                    }
                    const int n3 = cs3(LA, ia) + cs3(LB, ib) + cs3(LC, ic) + cs3(LD, id);
                    double v = (double)acc[((ia * NB + ib) * NC + ic) * ND + id];
                    if (n3 == 1) v *= s3;
                    else if (n3 == 2) v *= 3.0;
                    else if (n3 == 3) v *= 3.0 * s3;
                    else if (n3 == 4) v *= 9.0;
                    if (fabs(v) < cut) continue;
                    long long i1 = bfA + ia + 1, j1 = bfB + ib + 1, k1 = bfC + ic + 1, l1 = bfD + id + 1;
                    long long i2 = i1, j2 = j1, k2 = k1, l2 = l1;
                    if (i1 < j1) { i2 = j1; j2 = i1; }
                    if (k1 < l1) { k2 = l1; l2 = k1; }
                    long long ii = i2, jj = j2, kk = k2, ll = l2;
                    if (ii < kk) { ii = k2; jj = l2; kk = i2; ll = j2; }
                    else if (ii == kk && jj < ll) { jj = l2; ll = j2; }
                    if (ii == jj) v *= 0.5;
                    if (kk == ll) v *= 0.5;
                    if (ii == kk && jj == ll) v *= 0.5;
                    const long long ij = tri1(ii, jj) - 1, kl = tri1(kk, ll) - 1;
                    const long long ik = tri1(ii, kk) - 1, jl = tri1(jj, ll) - 1;
                    const long long il = tri1(ii, ll) - 1, jk = tri1(jj, kk) - 1;
                    const double v4 = 4.0 * v;
                    atomicAdd(F + ij, v4 * __ldg(Dm + kl));
                    atomicAdd(F + kl, v4 * __ldg(Dm + ij));
                    atomicAdd(F + ik, -v * __ldg(Dm + jl));
                    atomicAdd(F + jl, -v * __ldg(Dm + ik));
                    atomicAdd(F + il, -v * __ldg(Dm + jk));
                    atomicAdd(F + jk, -v * __ldg(Dm + il));
                }
        }
}

// ---- reference rank ownership (int0000.F90:76-91, int0001.F90:89-104) ---------
__device__ __forceinline__ bool rank_owns(const RankSplit &rs, long long it) {
    const long long ntot = rs.ntot;
    if (rs.tile == TILE_NONE) {
        long long nchunk = ntot / rs.nsize;
        long long s = nchunk * rs.rank + 1, e = s + nchunk - 1;
        if (rs.rank == rs.nsize - 1) e = ntot;
        return it >= s && it <= e;
    }
    long long chunk = rs.tile == TILE_SQRT ? 61237LL : (rs.tile == TILE_E9 ? 3750000000LL : 375000000LL);
    if (ntot <= chunk) chunk = ntot;
    long long ntile = ntot / chunk;
    long long t = (it - 1) / chunk + 1;
    if (t > ntile) t = ntile;
    long long is = (t - 1) * chunk + 1, ie = t * chunk;
    if (t == ntile) ie = ntot;
    long long nchunk = (ie - is) / rs.nsize;
    long long s = nchunk * rs.rank + is, e = s + nchunk - 1;
    if (rs.rank == rs.nsize - 1) e = ie;
    return it >= s && it <= e;
}

struct ClassArgs {
    DevBasis b;
    const double *tab;
    const double *Dm;
    double *F;
    double cut;
    double thr;
    bool strict;
    int nbra;
    const int *bra_ids, *ket_ids, *bra_orig, *ket_orig;
    const long long *pref;   // nbra+1
    const int *koff;         // per-bra first ket position (FP32 items) or null
    RankSplit rs;
};

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) class_kernel(ClassArgs a) {
    using Q = Quartet<LA, LB, LC, LD, R>;
    const long long total = a.pref[a.nbra];
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = a.nbra;
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (__ldg(a.pref + mid) <= g) lo = mid; else hi = mid;
        }
        const int i = lo;
        const int j = (int)(g - __ldg(a.pref + i)) + (a.koff ? __ldg(a.koff + i) : 0);
        if (a.rs.nsize > 1) {
            const long long bo = a.bra_orig[i], ko = a.ket_orig[j];
            long long it;
            if (a.rs.tri) it = (bo > ko ? bo : ko) + 1;
            else if (a.rs.ketmajor) it = ko * a.rs.nbra_ref + bo + 1;
            else it = bo * a.rs.nket_ref + ko + 1;
            if (!rank_owns(a.rs, it)) continue;
        }
        const int P = __ldg(a.bra_ids + i), Qd = __ldg(a.ket_ids + j);
        R acc[Q::NCART];
        Q::eval(a.b, P, Qd, a.thr, a.strict, a.tab, acc);
        const int2 sab = a.b.pair_shell[P], scd = a.b.pair_shell[Qd];
        digest<LA, LB, LC, LD, R>(acc, a.b.shell_bf0[sab.x], a.b.shell_bf0[sab.y],
                                  a.b.shell_bf0[scd.x], a.b.shell_bf0[scd.y], sab.x == sab.y,
                                  scd.x == scd.y, P == Qd, a.cut, a.Dm, a.F);
    }
}


template <int LA, int LB, int LC, int LD>
cudaError_t launch_t(const ClassArgs &a, long long work, int precision, int num_sms, cudaStream_t st) {
    if (work <= 0) return cudaSuccess;
    const int threads = 128;
    long long blocks = (work + threads - 1) / threads;
    long long cap = (long long)num_sms * 32;
    if (blocks > cap) blocks = cap;
    if (precision == 0)
        class_kernel<LA, LB, LC, LD, double><<<(unsigned)blocks, threads, 0, st>>>(a);
    else
        class_kernel<LA, LB, LC, LD, float><<<(unsigned)blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace liberi
