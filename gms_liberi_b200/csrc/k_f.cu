// k_f.cu -- the 34 f-shell quartet classes of the reference's ENABLE_F block
// (src/liberi_driver.F90:103-160: the ERIC kernels int0030/0031/0032/1030 and
// the generated Rys kernels, src/rhf/eric, src/rhf/rys).
//
// An f quartet is too large for the thread-per-quartet class kernels ((ff|ff)
// holds 10,000 integrals and 7 roots), so a group of threads evaluates one
// shell quartet at a time, everything in shared memory, with the class's
// angular momenta as compile-time parameters (one instantiation per class).
// The group is one warp (four tasks per CTA, warp barriers only) where the
// quartet's working set fits 24 KB, else a whole 256-thread CTA:
//   1. 3 n threads per primitive quartet (one per root and Cartesian axis)
//      take the root and weight from the 7-root table and run the 2D vertical
//      recurrence g[e][f], e <= la+lb, f <= lc+ld (prefactor and weight folded
//      into the x axis);
//   2. all threads expand g to the 2D integrals I[a][b][c][d] by the closed
//      form of the transfer relation, I = sum_i sum_k C(b,i) AB^(b-i) C(d,k)
//      CD^(d-k) g[a+i][c+k];
//   3. every thread accumulates its own Cartesian components of the shell
//      quartet, sum_r Ix Iy Iz, into the block in shared memory.
// Several primitive quartets share one round when shared memory allows.
// After the last primitive quartet every thread digests its own components
// with the DIRFCK rules (unique components for equal shells, 0.5 factors on
// equal functions, the six packed updates, src/rhf/rys/int3011_rysgen.F90
// digestion) by FP64 atomics, reading D from the build's full matrix.
// FP64 only: a mixed-precision build runs its f classes in FP64.
#include "quartet.cuh"

namespace liberi {

constexpr int FCLASS_THREADS = 128;

// Shared-memory bytes of one group of a class: the quartet's block, npq
// rounds' VRR and 2D-integral tables, the component index tables.
__host__ __device__ constexpr int fnc(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr size_t fgroup_bytes(int la, int lb, int lc, int ld, int npq) {
    return sizeof(double) * ((size_t)fnc(la) * fnc(lb) * fnc(lc) * fnc(ld) +
                             (size_t)npq * 3 * ((la + lb + lc + ld) / 2 + 1) *
                                 ((la + lb + 1) * (lc + ld + 1) + (la + 1) * (lb + 1) * (lc + 1) * (ld + 1))) +
           3 * (size_t)(fnc(la) * fnc(lb) + fnc(lc) * fnc(ld)) + 16;
}
// One warp per quartet where the working set of one primitive quartet per
// round fits 24 KB, else the whole CTA.
__host__ __device__ constexpr bool fwarp_mode(int la, int lb, int lc, int ld) {
    return fgroup_bytes(la, lb, lc, ld, 1) <= 24 * 1024;
}
// Primitive quartets per round: as many as the group's threads take in step 1
// (3 n each) within 12 KB per warp group (four CTAs of four warps per SM) or
// 48 KB per CTA group (four or more CTAs of eight warps per SM where the
// block allows: a round rarely fills many slots, uncontracted polarisation
// shells having one primitive each).
__host__ __device__ constexpr int fnpq(int la, int lb, int lc, int ld, int nt) {
    int npq = nt / (3 * ((la + lb + lc + ld) / 2 + 1));
    while (npq > 1 && fgroup_bytes(la, lb, lc, ld, npq) > (nt == 32 ? 12 * 1024 : 48 * 1024)) npq--;
    return npq < 1 ? 1 : npq;
}

// Compile-time shape of one class (engine orientation, la >= lb, lc >= ld) for
// groups of NT threads: one warp (CTAs of four warps) or a whole CTA of NT.
template <int LA, int LB, int LC, int LD, int NT>
struct FS {
    static constexpr int la = LA, lb = LB, lc = LC, ld = LD, nt = NT;
    static constexpr int block = NT == 32 ? FCLASS_THREADS : NT;
    static constexpr int nroot = (LA + LB + LC + LD) / 2 + 1;
    static constexpr int nb = fnc(LB), nc = fnc(LC), nd = fnc(LD);
    static constexpr int ncd = nc * nd, ncomp = fnc(LA) * nb * ncd;
    static constexpr int e1 = LA + LB + 1, f1 = LC + LD + 1;              // VRR extents
    static constexpr int nab2 = (LA + 1) * (LB + 1), ncd2 = (LC + 1) * (LD + 1);  // 2D index extents
    static constexpr int npq = fnpq(LA, LB, LC, LD, NT);
    static constexpr int group_doubles = (int)((fgroup_bytes(LA, LB, LC, LD, npq) + 15) / 16 * 2);
};

namespace {

// Cartesian exponents of component i of a shell of angular momentum l (GAMESS
// order: p x,y,z; d xx,yy,zz,xy,xz,yz; f xxx,yyy,zzz,xxy,xxz,xyy,yyz,xzz,yzz,xyz)
__constant__ unsigned char c_cart[4][10][3] = {
    {{0, 0, 0}},
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}},
    {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {1, 1, 1}}};
__device__ __forceinline__ void cart3(int l, int i, int &x, int &y, int &z) {
    x = c_cart[l][i][0];
    y = c_cart[l][i][1];
    z = c_cart[l][i][2];
}

// per-component normalisation relative to the axial component: sqrt3 on the
// mixed d, sqrt5 on the six mixed f and sqrt15 on xyz (int3011_rysgen.F90 d03bra)
__device__ __forceinline__ double cnorm(int l, int i) {
    if (l == 2) return i >= 3 ? 1.7320508075688772935 : 1.0;
    if (l == 3) return i == 9 ? 3.8729833462074168852 : (i >= 3 ? 2.2360679774997896964 : 1.0);
    return 1.0;
}

__device__ __forceinline__ unsigned ftri(unsigned i, unsigned j) {
    return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

// root r and weight of the n-root Rys rule at T (large-T limit above thr,
// strict: T > thr, else T >= thr; always at and above the table's end)
__device__ __forceinline__ void rys7_root(int n, int r, double T, double thr, bool strict, const double *tab,
                                          double &u, double &w) {
    const bool asym = (strict ? (T > thr) : (T >= thr)) || T >= RYS7_TMAX;
    if (asym) {
        const double it = 1.0 / T;
        const double *hr = tab + rys7_herm_off(n);
        u = __ldg(hr + r) * it;
        w = __ldg(hr + MAXROOT7 + r) * sqrt(it);
        return;
    }
    const double t4 = T * (double)RYS_PER_UNIT;
    const int k = (int)t4;
    const double x = 2.0 * (t4 - (double)k) - 1.0, x2 = x * x, x4 = x2 * x2;
    const double *base = tab + rys7_table_off(n) + (size_t)k * (2 * n * RYS_NCOEF);
    double v[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const double *c = base + (h ? n + r : r) * RYS_NCOEF;
        const double a0 = fma(__ldg(c + 1), x, __ldg(c + 0)), a1 = fma(__ldg(c + 3), x, __ldg(c + 2));
        const double a2 = fma(__ldg(c + 5), x, __ldg(c + 4)), a3 = fma(__ldg(c + 7), x, __ldg(c + 6));
        v[h] = fma(fma(a3, x2, a2), x4, fma(a1, x2, a0));
    }
    u = v[0];
    w = v[1];
}

}  // namespace

// A group of NT threads evaluates one quartet at a time: a whole CTA (NT = 128)
// for the classes with large blocks, one warp (NT = 32) for the others, four
// warps of a CTA then working on four tasks with their own shared memory and
// warp barriers only.
template <int NT>
__device__ __forceinline__ int group_rank() { return NT == 32 ? (int)(threadIdx.x & 31) : (int)threadIdx.x; }
template <int NT>
__device__ __forceinline__ void group_sync() {
    if constexpr (NT == 32) __syncwarp();
    else __syncthreads();
}

// Shared-memory layout of one group: the quartet's block, the VRR tables and
// the 2D-integral tables of a round, and per component the 2D index on each axis.
struct FSmem {
    double *acc;         // [ncomp]
    double *g;           // [npq][3n][e1*f1]
    double *G;           // [npq][3n][nab2*ncd2]
    unsigned char *gab;  // [3][na*nb]: a*(lb+1)+b per axis
    unsigned char *gcd;  // [3][ncd]: c*(ld+1)+d per axis
    int nab;
};

// Carves the layout, fills the index tables and zeroes the block (the caller
// synchronises the group before use).
template <typename S>
__device__ __forceinline__ FSmem fsmem_setup(const S &s, double *fsm) {
    constexpr int NT = S::nt;
    FSmem m;
    const int tid = group_rank<NT>(), nrx = 3 * s.nroot;
    m.acc = fsm;
    m.g = m.acc + s.ncomp;
    m.G = m.g + (size_t)s.npq * nrx * s.e1 * s.f1;
    m.gab = reinterpret_cast<unsigned char *>(m.G + (size_t)s.npq * nrx * s.nab2 * s.ncd2);
    m.nab = s.ncomp / s.ncd;
    m.gcd = m.gab + 3 * m.nab;
    for (int i = tid; i < m.nab; i += NT) {
        int ax, ay, az, bx, by, bz;
        cart3(s.la, i / s.nb, ax, ay, az);
        cart3(s.lb, i % s.nb, bx, by, bz);
        m.gab[i] = (unsigned char)(ax * (s.lb + 1) + bx);
        m.gab[m.nab + i] = (unsigned char)(ay * (s.lb + 1) + by);
        m.gab[2 * m.nab + i] = (unsigned char)(az * (s.lb + 1) + bz);
    }
    for (int i = tid; i < s.ncd; i += NT) {
        int cx, cy, cz, dx, dy, dz;
        cart3(s.lc, i / s.nd, cx, cy, cz);
        cart3(s.ld, i % s.nd, dx, dy, dz);
        m.gcd[i] = (unsigned char)(cx * (s.ld + 1) + dx);
        m.gcd[s.ncd + i] = (unsigned char)(cy * (s.ld + 1) + dy);
        m.gcd[2 * s.ncd + i] = (unsigned char)(cz * (s.ld + 1) + dz);
    }
    for (int c = tid; c < s.ncomp; c += NT) m.acc[c] = 0.0;
    return m;
}

// Adds the contracted block of the quartet (P|Q) (pair P = (A,B), Q = (C,D))
// to m.acc: every thread keeps its own components c = rank + k * NT.  Called
// by the whole group; every round of primitive quartets ends with a group
// barrier, so the tables may be reused on return.
template <typename S>
__device__ __forceinline__ void fquartet_block(const S &s, const FSmem &m, const DevBasis &b, int P, int Q,
                                               double thr, bool strict, const double *__restrict__ tab7) {
    constexpr int NT = S::nt;
    const int tid = group_rank<NT>();
    const int n = s.nroot, nrx = 3 * n;
    const int gsz = s.e1 * s.f1;      // one VRR table
    const int Gsz = s.nab2 * s.ncd2;  // one 2D-integral table
    double *g = m.g, *G = m.G;
    const int nab = m.nab;
    const unsigned char *gab = m.gab, *gcd = m.gcd;
    const int2 sab = b.pair_shell[P], scd = b.pair_shell[Q];
    const double4 A = b.shell_xyz[sab.x], B = b.shell_xyz[sab.y];
    const double4 C = b.shell_xyz[scd.x], D = b.shell_xyz[scd.y];
    const int p0 = b.pair_prim0[P], np = b.pair_nprim[P];
    const int q0 = b.pair_prim0[Q], nq = b.pair_nprim[Q];
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const double CD[3] = {C.x - D.x, C.y - D.y, C.z - D.z};
    const int npq_total = np * nq;
    for (int pq0 = 0; pq0 < npq_total; pq0 += s.npq) {
        // slots of this round that hold a primitive quartet (uncontracted
        // polarisation shells leave most of them empty): steps 2 and 3 cover
        // only these
        const int nslot = min(s.npq, npq_total - pq0);
        // 1. roots and the vertical recurrence, one thread per (slot, root, axis)
        if (tid < nslot * nrx) {
            const int slot = tid / nrx, rx = tid - slot * nrx;
            const int r = rx / 3, x = rx - 3 * r;
            const int pq = pq0 + slot;
            double *gs = g + (size_t)(slot * nrx + rx) * gsz;
            if (pq < npq_total) {
                const int ip = pq / nq, iq = pq - ip * nq;
                const double4 Pp = b.prim_P[p0 + ip], Qp = b.prim_P[q0 + iq];
                const double2 Xp = b.prim_X[p0 + ip], Xq = b.prim_X[q0 + iq];
                const double p = Pp.w, q = Qp.w, ipq = 1.0 / (p + q);
                const double dx = Pp.x - Qp.x, dy = Pp.y - Qp.y, dz = Pp.z - Qp.z;
                const double T = p * q * ipq * (dx * dx + dy * dy + dz * dz);
                double u, w;
                rys7_root(n, r, T, thr, strict, tab7, u, w);
                const double B00 = 0.5 * u * ipq;
                const double B10 = 0.5 / p * (1.0 - q * u * ipq);
                const double B01 = 0.5 / q * (1.0 - p * u * ipq);
                const double PA = x == 0 ? Pp.x - A.x : (x == 1 ? Pp.y - A.y : Pp.z - A.z);
                const double QC = x == 0 ? Qp.x - C.x : (x == 1 ? Qp.y - C.y : Qp.z - C.z);
                const double PQ = x == 0 ? dx : (x == 1 ? dy : dz);
                const double C00 = PA - q * u * ipq * PQ;
                const double Cp00 = QC + p * u * ipq * PQ;
                const double g00 = x == 0 ? Xp.x * Xq.x * sqrt(ipq) * w : 1.0;
                const int e1 = s.e1, f1 = s.f1;
                gs[0] = g00;
                for (int e = 0; e + 1 < e1; e++) {
                    double v = C00 * gs[e * f1];
                    if (e > 0) v += (double)e * B10 * gs[(e - 1) * f1];
                    gs[(e + 1) * f1] = v;
                }
                for (int f = 0; f + 1 < f1; f++)
                    for (int e = 0; e < e1; e++) {
                        double v = Cp00 * gs[e * f1 + f];
                        if (f > 0) v += (double)f * B01 * gs[e * f1 + f - 1];
                        if (e > 0) v += (double)e * B00 * gs[(e - 1) * f1 + f];
                        gs[e * f1 + f + 1] = v;
                    }
            }
        }
        group_sync<NT>();
        // 2. transfer to the 2D integrals of every (slot, root, axis)
        const int nG = nslot * nrx * Gsz;
        for (int idx = tid; idx < nG; idx += NT) {
            const int tab_i = idx / Gsz, rem = idx - tab_i * Gsz;
            const int x = tab_i % 3;
            const int iab = rem / s.ncd2, icd = rem - iab * s.ncd2;
            const int ia = iab / (s.lb + 1), ib = iab - ia * (s.lb + 1);
            const int ic = icd / (s.ld + 1), id = icd - ic * (s.ld + 1);
            const double ab = AB[x], cd = CD[x];
            const double *gs = g + (size_t)tab_i * gsz;
            // i, k from the top: weights C(ib,i) AB^(ib-i) and C(id,k) CD^(id-k),
            // the binomial updated as C(n,m-1) = C(n,m) m / (n-m+1)
            double sum = 0.0, wb = 1.0;
            for (int i = ib; i >= 0; i--) {
                double inner = 0.0, wd = 1.0;
                for (int k = id; k >= 0; k--) {
                    inner = fma(wd, gs[(ia + i) * s.f1 + ic + k], inner);
                    wd *= cd * (double)k / (double)(id - k + 1);
                }
                sum = fma(wb, inner, sum);
                wb *= ab * (double)i / (double)(ib - i + 1);
            }
            G[idx] = sum;
        }
        group_sync<NT>();
        // 3. assembly: every thread its own components
        for (int c = tid; c < s.ncomp; c += NT) {
            const int iab = c / s.ncd, icd = c - iab * s.ncd;
            const int ix = gab[iab] * s.ncd2 + gcd[icd];
            const int iy = gab[nab + iab] * s.ncd2 + gcd[s.ncd + icd];
            const int iz = gab[2 * nab + iab] * s.ncd2 + gcd[2 * s.ncd + icd];
            double v = 0.0;
            const int ntab = nslot * n;
            for (int tr = 0; tr < ntab; tr++) {
                const double *Gt = G + (size_t)tr * 3 * Gsz;
                v = fma(Gt[ix] * Gt[Gsz + iy], Gt[2 * Gsz + iz], v);
            }
            m.acc[c] += v;
        }
        group_sync<NT>();
    }
}

// NT = 256: one task per CTA; NT = 32: one task per warp (four per CTA).
template <typename S>
__global__ void __launch_bounds__(S::block) fclass_kernel(ClassArgs a, const double *__restrict__ tab7) {
    constexpr int NT = S::nt;
    constexpr S s{};
    constexpr int GROUPS = S::block / NT;
    const int grp = NT == 32 ? (int)(threadIdx.x >> 5) : 0;
    const int task = (int)blockIdx.x * GROUPS + grp;
    if (task >= a.ntasks) return;  // the whole group (only warp barriers follow in warp mode)
    extern __shared__ __align__(16) double fsm[];
    const int tid = group_rank<NT>();
    const FSmem m = fsmem_setup(s, fsm + (size_t)grp * s.group_doubles);
    double *acc = m.acc;
    group_sync<NT>();

    const int4 t = a.tasks[task];
    const DevBasis &b = a.b;
    const int P = a.bra_ids[t.x];
    const int2 sab = b.pair_shell[P];
    const int bfA = b.shell_bf0[sab.x], bfB = b.shell_bf0[sab.y];
    const unsigned nbf = (unsigned)a.nbf;
    const double *Dm = a.Dm, *Dk = a.Dm + a.k_offset;

    for (int qi = 0; qi < t.z; qi++) {
        const int j = t.y + qi;
        if (a.rs.nsize > 1 && !quartet_owned(a, t.x, j)) continue;  // uniform over the group
        const int Q = a.ket_ids[j];
        const int2 scd = b.pair_shell[Q];
        const int bfC = b.shell_bf0[scd.x], bfD = b.shell_bf0[scd.y];
        fquartet_block(s, m, b, P, Q, a.thr, a.strict, tab7);
        // digestion of this thread's components (the same components it
        // accumulated: no barrier needed before the reads)
        const bool iandj = sab.x == sab.y, kandl = scd.x == scd.y;
        const bool same = sab.x == scd.x && sab.y == scd.y;
        for (int c = tid; c < s.ncomp; c += NT) {
            double val = acc[c];
            acc[c] = 0.0;
            const int iab = c / s.ncd, icd = c - iab * s.ncd;
            const int ia = iab / s.nb, ib = iab - ia * s.nb;
            const int ic = icd / s.nd, id = icd - ic * s.nd;
            if (iandj && ib > ia) continue;
            if (kandl && id > ic) continue;
            if (same) {
                const int pij = iandj ? ia * (ia + 1) / 2 + ib : ia * s.nb + ib;
                const int pkl = kandl ? ic * (ic + 1) / 2 + id : ic * s.nd + id;
                if (pkl > pij) continue;
            }
            val *= cnorm(s.la, ia) * cnorm(s.lb, ib) * cnorm(s.lc, ic) * cnorm(s.ld, id);
            if (fabs(val) < a.cut) continue;
            unsigned i2 = bfA + ia, j2 = bfB + ib, k2 = bfC + ic, l2 = bfD + id;
            if (i2 < j2) { const unsigned tt = i2; i2 = j2; j2 = tt; }
            if (k2 < l2) { const unsigned tt = k2; k2 = l2; l2 = tt; }
            unsigned ii = i2, jj = j2, kk = k2, ll = l2;
            if (ii < kk || (ii == kk && jj < ll)) { ii = k2; jj = l2; kk = i2; ll = j2; }
            if (ii == jj) val *= 0.5;
            if (kk == ll) val *= 0.5;
            if (ii == kk && jj == ll) val *= 0.5;
            const double v4 = 4.0 * val;
            atomicAdd(a.F + ftri(ii, jj), v4 * Dm[kk * nbf + ll]);
            atomicAdd(a.F + ftri(kk, ll), v4 * Dm[ii * nbf + jj]);
            atomicAdd(a.F + ftri(ii, kk), -val * Dk[jj * nbf + ll]);
            atomicAdd(a.F + ftri(jj, ll), -val * Dk[ii * nbf + kk]);
            atomicAdd(a.F + ftri(ii, ll), -val * Dk[jj * nbf + kk]);
            atomicAdd(a.F + ftri(jj, kk), -val * Dk[ii * nbf + ll]);
        }
    }
}

// Schwarz values of f pairs: one CTA per pair P of one class, the (P|P) block
// as in the class kernel, then sqrt(max over components |(ab|ab)|) of the
// normalised integrals into out[P] (global pair index).
template <typename S>
__global__ void __launch_bounds__(FCLASS_THREADS) fschwarz_kernel(DevBasis b, int pair_off, int npairs,
                                                                  const double *__restrict__ tab7, double *out) {
    if ((int)blockIdx.x >= npairs) return;
    constexpr S s{};
    static_assert(S::nt == FCLASS_THREADS, "one pair per CTA");
    extern __shared__ __align__(16) double fsm[];
    __shared__ double wmax[FCLASS_THREADS / 32];
    const FSmem m = fsmem_setup(s, fsm);
    __syncthreads();
    const int P = pair_off + (int)blockIdx.x;
    fquartet_block(s, m, b, P, P, RYS7_TMAX, false, tab7);
    // diagonal components (a b|a b): icd == iab
    double mx = 0.0;
    for (int iab = threadIdx.x; iab < m.nab; iab += FCLASS_THREADS) {
        const int ia = iab / s.nb, ib = iab - ia * s.nb;
        const double nrm = cnorm(s.la, ia) * cnorm(s.lb, ib);
        mx = fmax(mx, fabs(m.acc[iab * s.ncd + iab]) * nrm * nrm);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < FCLASS_THREADS / 32; w++) mx = fmax(mx, wmax[w]);
        out[P] = sqrt(mx);
    }
}

template <int LF>
static cudaError_t fschwarz_t(int npairs, int pair_off, const DevBasis &b, const double *tab7, double *out,
                              cudaStream_t stream) {
    using S = FS<3, LF, 3, LF, FCLASS_THREADS>;
    const size_t smem = (size_t)S::group_doubles * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(fschwarz_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fschwarz_kernel<S><<<(unsigned)npairs, FCLASS_THREADS, smem, stream>>>(b, pair_off, npairs, tab7, out);
    return cudaGetLastError();
}

cudaError_t launch_fschwarz(int pair_class, int npairs, int pair_off, const DevBasis &b, const double *rys_tab7,
                            double *out, cudaStream_t stream) {
    if (npairs <= 0) return cudaSuccess;
    if (!rys_tab7) return cudaErrorInvalidValue;
    switch (pair_class) {  // sf, pf, df, ff: the lower-L shell s, p, d, f
        case SF: return fschwarz_t<0>(npairs, pair_off, b, rys_tab7, out, stream);
        case PF: return fschwarz_t<1>(npairs, pair_off, b, rys_tab7, out, stream);
        case DF: return fschwarz_t<2>(npairs, pair_off, b, rys_tab7, out, stream);
        case FF: return fschwarz_t<3>(npairs, pair_off, b, rys_tab7, out, stream);
        default: return cudaErrorInvalidValue;
    }
}

// one class: warp or CTA groups by its shape, one launch over the plan's tasks
template <int LA, int LB, int LC, int LD>
static cudaError_t fclass_t(const ClassArgs &a, const double *tab7, cudaStream_t stream) {
    constexpr bool W = fwarp_mode(LA, LB, LC, LD);
    using S = FS<LA, LB, LC, LD, W ? 32 : 2 * FCLASS_THREADS>;
    constexpr int groups = S::block / S::nt;
    const size_t smem = (size_t)groups * S::group_doubles * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(fclass_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)((a.ntasks + groups - 1) / groups);
    fclass_kernel<S><<<grid, S::block, smem, stream>>>(a, tab7);
    return cudaGetLastError();
}

cudaError_t launch_fclass(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs, int nbf) {
    if (plan.ntasks <= 0) return cudaSuccess;
    const KernelDesc &kd = KDESC[k];
    ClassArgs a{};
    a.b = ctx.basis;
    a.Dm = ctx.D;
    a.F = ctx.F;
    a.cut = kd.digest_schwarz ? ctx.schwarz_cut : ctx.eri_cut;
    a.thr = kd.asym;
    a.strict = !kd.rys;
    a.tasks = plan.tasks;
    a.ntasks_dev = nullptr;
    a.ntasks = plan.ntasks;
    a.nbf = nbf;
    a.bra_ids = plan.bra_ids;
    a.ket_ids = plan.ket_ids;
    a.bra_orig = plan.bra_orig;
    a.ket_orig = plan.ket_orig;
    a.ket_rec = plan.ket_rec;
    a.swapped = plan.swapped;
    a.rs = rs;
    a.k_offset = ctx.k_offset;
    // the engine orientation (la lb lc ld) of classes 21..54, KDESC order
#define LIBERI_F(kk, A, B, C, D) \
    case kk: return fclass_t<A, B, C, D>(a, ctx.rys_tab7, ctx.stream);
    switch (k) {
        LIBERI_F(21, 3, 3, 3, 3) LIBERI_F(22, 0, 0, 3, 0) LIBERI_F(23, 0, 0, 3, 1) LIBERI_F(24, 0, 0, 3, 2)
        LIBERI_F(25, 1, 0, 3, 0) LIBERI_F(26, 3, 3, 3, 0) LIBERI_F(27, 3, 0, 1, 1) LIBERI_F(28, 3, 0, 2, 0)
        LIBERI_F(29, 2, 1, 3, 0) LIBERI_F(30, 2, 2, 3, 0) LIBERI_F(31, 3, 0, 3, 0) LIBERI_F(32, 3, 1, 1, 0)
        LIBERI_F(33, 3, 1, 1, 1) LIBERI_F(34, 3, 1, 2, 0) LIBERI_F(35, 3, 1, 2, 1) LIBERI_F(36, 2, 2, 3, 1)
        LIBERI_F(37, 3, 1, 3, 0) LIBERI_F(38, 3, 1, 3, 1) LIBERI_F(39, 3, 2, 1, 0) LIBERI_F(40, 3, 3, 3, 1)
        LIBERI_F(41, 3, 2, 1, 1) LIBERI_F(42, 3, 2, 2, 0) LIBERI_F(43, 3, 2, 2, 1) LIBERI_F(44, 3, 2, 2, 2)
        LIBERI_F(45, 3, 2, 3, 0) LIBERI_F(46, 3, 2, 3, 1) LIBERI_F(47, 3, 2, 3, 2) LIBERI_F(48, 3, 3, 0, 0)
        LIBERI_F(49, 3, 3, 1, 0) LIBERI_F(50, 3, 3, 1, 1) LIBERI_F(51, 3, 3, 2, 0) LIBERI_F(52, 3, 3, 2, 1)
        LIBERI_F(53, 3, 3, 2, 2) LIBERI_F(54, 3, 3, 3, 2)
        default: return cudaErrorInvalidValue;
    }
#undef LIBERI_F
}

}  // namespace liberi
