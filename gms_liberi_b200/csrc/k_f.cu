// k_f.cu -- the 34 f-shell quartet classes of the reference's ENABLE_F block
// (src/liberi_driver.F90:103-160: the ERIC kernels int0030/0031/0032/1030 and
// the generated Rys kernels, src/rhf/eric, src/rhf/rys).
//
// An f quartet is too large for the thread-per-quartet class kernels ((ff|ff)
// holds 10,000 integrals and 7 roots), so one CTA evaluates one shell quartet
// at a time, everything in shared memory, with the class's angular momenta as
// run-time parameters (one kernel serves all 34 classes):
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

struct FShape {
    int la, lb, lc, ld;  // engine orientation (la >= lb, lc >= ld)
    int nroot;
    int nb, nc, nd;      // Cartesian components of B, C, D
    int ncd, ncomp;      // nc * nd, na * nb * nc * nd
    int e1, f1;          // VRR extents la+lb+1, lc+ld+1
    int nab2, ncd2;      // 2D index extents (la+1)(lb+1), (lc+1)(ld+1)
    int npq;             // primitive quartets per round
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

__global__ void __launch_bounds__(FCLASS_THREADS) fclass_kernel(ClassArgs a, const double *__restrict__ tab7,
                                                                FShape s) {
    if ((int)blockIdx.x >= a.ntasks) return;
    extern __shared__ __align__(16) double fsm[];
    const int tid = threadIdx.x;
    const int n = s.nroot, nrx = 3 * n;
    const int gsz = s.e1 * s.f1;          // one VRR table
    const int Gsz = s.nab2 * s.ncd2;      // one 2D-integral table
    double *acc = fsm;                          // [ncomp]
    double *g = acc + s.ncomp;                  // [npq][3n][e1*f1]
    double *G = g + (size_t)s.npq * nrx * gsz;  // [npq][3n][nab2*ncd2]
    // component -> 2D index per axis: AB part (a*(lb+1)+b), CD part (c*(ld+1)+d)
    unsigned char *gab = reinterpret_cast<unsigned char *>(G + (size_t)s.npq * nrx * Gsz);  // [3][na*nb]
    const int nab = s.ncomp / s.ncd;
    unsigned char *gcd = gab + 3 * nab;  // [3][ncd]
    for (int i = tid; i < nab; i += FCLASS_THREADS) {
        int ax, ay, az, bx, by, bz;
        cart3(s.la, i / s.nb, ax, ay, az);
        cart3(s.lb, i % s.nb, bx, by, bz);
        gab[i] = (unsigned char)(ax * (s.lb + 1) + bx);
        gab[nab + i] = (unsigned char)(ay * (s.lb + 1) + by);
        gab[2 * nab + i] = (unsigned char)(az * (s.lb + 1) + bz);
    }
    for (int i = tid; i < s.ncd; i += FCLASS_THREADS) {
        int cx, cy, cz, dx, dy, dz;
        cart3(s.lc, i / s.nd, cx, cy, cz);
        cart3(s.ld, i % s.nd, dx, dy, dz);
        gcd[i] = (unsigned char)(cx * (s.ld + 1) + dx);
        gcd[s.ncd + i] = (unsigned char)(cy * (s.ld + 1) + dy);
        gcd[2 * s.ncd + i] = (unsigned char)(cz * (s.ld + 1) + dz);
    }
    for (int c = tid; c < s.ncomp; c += FCLASS_THREADS) acc[c] = 0.0;
    __syncthreads();

    const int4 t = a.tasks[blockIdx.x];
    const DevBasis &b = a.b;
    const int P = a.bra_ids[t.x];
    const int2 sab = b.pair_shell[P];
    const double4 A = b.shell_xyz[sab.x], B = b.shell_xyz[sab.y];
    const int bfA = b.shell_bf0[sab.x], bfB = b.shell_bf0[sab.y];
    const int p0 = b.pair_prim0[P], np = b.pair_nprim[P];
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    const unsigned nbf = (unsigned)a.nbf;
    const double *Dm = a.Dm, *Dk = a.Dm + a.k_offset;

    for (int qi = 0; qi < t.z; qi++) {
        const int j = t.y + qi;
        if (a.rs.nsize > 1 && !quartet_owned(a, t.x, j)) continue;  // uniform over the CTA
        const int Q = a.ket_ids[j];
        const int2 scd = b.pair_shell[Q];
        const double4 C = b.shell_xyz[scd.x], D = b.shell_xyz[scd.y];
        const int bfC = b.shell_bf0[scd.x], bfD = b.shell_bf0[scd.y];
        const int q0 = b.pair_prim0[Q], nq = b.pair_nprim[Q];
        const double CD[3] = {C.x - D.x, C.y - D.y, C.z - D.z};
        const int npq_total = np * nq;
        for (int pq0 = 0; pq0 < npq_total; pq0 += s.npq) {
            // 1. roots and the vertical recurrence, one thread per (slot, root, axis)
            if (tid < s.npq * nrx) {
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
                    rys7_root(n, r, T, a.thr, a.strict, tab7, u, w);
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
                } else {
                    for (int i = 0; i < gsz; i++) gs[i] = 0.0;  // empty slot contributes nothing
                }
            }
            __syncthreads();
            // 2. transfer to the 2D integrals of every (slot, root, axis)
            const int nG = s.npq * nrx * Gsz;
            for (int idx = tid; idx < nG; idx += FCLASS_THREADS) {
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
            __syncthreads();
            // 3. assembly: every thread its own components
            for (int c = tid; c < s.ncomp; c += FCLASS_THREADS) {
                const int iab = c / s.ncd, icd = c - iab * s.ncd;
                const int ix = gab[iab] * s.ncd2 + gcd[icd];
                const int iy = gab[nab + iab] * s.ncd2 + gcd[s.ncd + icd];
                const int iz = gab[2 * nab + iab] * s.ncd2 + gcd[2 * s.ncd + icd];
                double v = 0.0;
                const int ntab = s.npq * n;
                for (int tr = 0; tr < ntab; tr++) {
                    const double *Gt = G + (size_t)tr * 3 * Gsz;
                    v = fma(Gt[ix] * Gt[Gsz + iy], Gt[2 * Gsz + iz], v);
                }
                acc[c] += v;
            }
            __syncthreads();
        }
        // digestion of this thread's components (the same components it
        // accumulated: no barrier needed before the reads)
        const bool iandj = sab.x == sab.y, kandl = scd.x == scd.y;
        const bool same = sab.x == scd.x && sab.y == scd.y;
        for (int c = tid; c < s.ncomp; c += FCLASS_THREADS) {
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

// shared-memory bytes of one CTA of this shape
static size_t fclass_smem(const FShape &s) {
    const size_t nab = (size_t)s.ncomp / s.ncd;
    return sizeof(double) * ((size_t)s.ncomp + (size_t)s.npq * 3 * s.nroot * (s.e1 * s.f1 + s.nab2 * s.ncd2)) +
           3 * (nab + s.ncd) + 16;
}

static FShape fshape_of(const KernelDesc &kd) {
    FShape s;
    s.la = kd.la;
    s.lb = kd.lb;
    s.lc = kd.lc;
    s.ld = kd.ld;
    s.nroot = (s.la + s.lb + s.lc + s.ld) / 2 + 1;
    const int na = (s.la + 1) * (s.la + 2) / 2;
    s.nb = (s.lb + 1) * (s.lb + 2) / 2;
    s.nc = (s.lc + 1) * (s.lc + 2) / 2;
    s.nd = (s.ld + 1) * (s.ld + 2) / 2;
    s.ncd = s.nc * s.nd;
    s.ncomp = na * s.nb * s.ncd;
    s.e1 = s.la + s.lb + 1;
    s.f1 = s.lc + s.ld + 1;
    s.nab2 = (s.la + 1) * (s.lb + 1);
    s.ncd2 = (s.lc + 1) * (s.ld + 1);
    // as many primitive quartets per round as the threads of step 1 and a
    // 96 KB shared-memory budget allow (two CTAs per SM)
    s.npq = FCLASS_THREADS / (3 * s.nroot);
    while (s.npq > 1) {
        if (fclass_smem(s) <= 96 * 1024) break;
        s.npq--;
    }
    return s;
}

size_t fclass_smem_bytes(int k) { return fclass_smem(fshape_of(KDESC[k])); }

cudaError_t launch_fclass(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs, int nbf) {
    if (plan.ntasks <= 0) return cudaSuccess;
    const KernelDesc &kd = KDESC[k];
    const FShape s = fshape_of(kd);
    const size_t smem = fclass_smem(s);
    cudaError_t e = cudaFuncSetAttribute(fclass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
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
    fclass_kernel<<<(unsigned)plan.ntasks, FCLASS_THREADS, smem, ctx.stream>>>(a, ctx.rys_tab7, s);
    return cudaGetLastError();
}

}  // namespace liberi
