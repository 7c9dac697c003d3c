// kernels.cu -- class dispatch, Schwarz generator and mixed-precision task
// builder of the Fock-build engine; the class kernels themselves are
// instantiated in k_*.cu from quartet.cuh.
#include "quartet.cuh"

namespace liberi {


#define LIBERI_CLASSES(X)                                                                    \
    X(0, 0, 0, 0, 0) X(1, 1, 0, 0, 0) X(2, 1, 1, 0, 0) X(3, 1, 1, 1, 0) X(4, 1, 0, 1, 0)         \
    X(5, 1, 1, 1, 1) X(6, 2, 0, 0, 0) X(7, 2, 1, 0, 0) X(8, 2, 0, 1, 0) X(9, 2, 1, 1, 0)         \
    X(10, 2, 2, 0, 0) X(11, 2, 2, 1, 0) X(12, 1, 1, 2, 0) X(13, 2, 0, 2, 0) X(14, 2, 2, 1, 1)    \
    X(15, 2, 1, 2, 1) X(16, 2, 1, 2, 0) X(17, 2, 1, 1, 1) X(18, 2, 2, 2, 0) X(19, 2, 2, 2, 1)    \
    X(20, 2, 2, 2, 2)

#define LIBERI_EXTERN(k, a, b, c, d) \
    extern template cudaError_t launch_t<a, b, c, d>(const ClassArgs &, int, int, cudaStream_t);
LIBERI_CLASSES(LIBERI_EXTERN)

// Schwarz table: sqrt(max |(ab|ab)|) per pair of one class
template <int LA, int LB>
__global__ void __launch_bounds__(64) schwarz_kernel(DevBasis b, int pair_off, int npairs,
                                                     const double *tab, double *out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int P = pair_off + t;
    out[t] = schwarz_diag<LA, LB>(b, P, tab, b.pair_prim0[P], b.pair_nprim[P]);
}

// Primitive-pair bounds: for every kept primitive pair k of pair P,
// sqrt(max |(ab|ab)|) of that primitive alone (with its contraction
// coefficients), rounded up to float: |(ab|cd)_prim| <= out[k] * out[l].
template <int LA, int LB>
__global__ void __launch_bounds__(64) prim_bound_kernel(DevBasis b, int pair_off, int npairs, const double *tab,
                                                        float *out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int P = pair_off + t;
    const int p0 = b.pair_prim0[P], np = b.pair_nprim[P];
    for (int k = p0; k < p0 + np; k++) {
        const double v = schwarz_diag<LA, LB>(b, P, tab, k, 1);
        out[k] = __double2float_ru(v * (1.0 + 1e-6));
    }
}

__global__ void maxabs_kernel(const double *x, long long n, unsigned long long *out) {
    double m = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Per plan item (bra, ket segment, surviving count): split = number of its
// kets with x_bra*x_ket*max|D| >= fp32_cut (a prefix, the segment is sorted
// by x); FP64 tasks cover [0, split), FP32 tasks [split, count).  One CTA
// builds both task lists; counts[0..1] are the task counts, counts[2..3] the
// FP32 quartet count (low, high word).
__device__ __forceinline__ int item_split(const int4 &it, const double *bra_x, const double *ket_x, double maxd,
                                          double fp32_cut) {
    const double xb = bra_x[it.x];
    int lo = 0, hi = it.z;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (xb * ket_x[it.y + mid] * maxd >= fp32_cut) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// One thread per item: the split point, then output ranges reserved with
// atomics (task order only affects load balance).  counts[0..1]: FP64 and
// FP32 task counts, counts[2..3]: FP32 quartet count (64-bit, low word first);
// zeroed before the launch.  BATCH: item.w is the molecule, whose Schwarz
// lists and max|D| are used and which the tasks carry; else one molecule.
template <bool BATCH>
__global__ void __launch_bounds__(256) split_tasks_kernel(int nitems, const int4 *items, const double *bra_x1,
                                                          const double *ket_x1, const ClassView *cviews,
                                                          const unsigned long long *maxd_bits, double fp32_cut,
                                                          int chunk, int4 *tasks64, int4 *tasks32, int *counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    const int4 it = items[i];
    const double *bx = BATCH ? cviews[it.w].bra_x : bra_x1;
    const double *kx = BATCH ? cviews[it.w].ket_x : ket_x1;
    const double maxd = __longlong_as_double((long long)maxd_bits[BATCH ? it.w : 0]);
    const int s = item_split(it, bx, kx, maxd, fp32_cut);
    const int n64 = (s + chunk - 1) / chunk, n32 = (it.z - s + chunk - 1) / chunk;
    const int w = BATCH ? it.w : 0;
    if (n64) {
        int o = atomicAdd(counts, n64);
        for (int k = 0; k < s; k += chunk) tasks64[o++] = make_int4(it.x, it.y + k, min(chunk, s - k), w);
    }
    if (n32) {
        int o = atomicAdd(counts + 1, n32);
        for (int k = s; k < it.z; k += chunk) tasks32[o++] = make_int4(it.x, it.y + k, min(chunk, it.z - k), w);
        atomicAdd(reinterpret_cast<unsigned long long *>(counts + 2), (unsigned long long)(it.z - s));
    }
}

cudaError_t launch_prim_bound(int pc, int npairs, int pair_off, const DevBasis &b, const double *tab, float *out,
                              cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    const int threads = 64;
    const unsigned blocks = (unsigned)((npairs + threads - 1) / threads);
    switch (pc) {
        case SS: prim_bound_kernel<0, 0><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case SP: prim_bound_kernel<1, 0><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case PP: prim_bound_kernel<1, 1><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case SD: prim_bound_kernel<2, 0><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case PD: prim_bound_kernel<2, 1><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case DD: prim_bound_kernel<2, 2><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ---- fingerprint of the evaluated quartet set -------------------------------------
// Per class {count, sum, xor} of a 64-bit hash of every quartet a launch over
// the same task list evaluates: the task walk and the rank-ownership test of
// class_task, the quartet's shells from the plan's pair ids.  The hash is
// the oracle's quartet_fp (oracle/liberi_oracle.c): unordered shell pairs,
// unordered pair of pairs, one 64-bit mix; sum and xor do not depend on the
// order of evaluation.
__device__ __forceinline__ unsigned long long fp_mix64(unsigned long long x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}
__device__ __forceinline__ unsigned long long quartet_fp(int2 ab, int2 cd) {
    const unsigned long long a = (unsigned)ab.x, b = (unsigned)ab.y, c = (unsigned)cd.x, d = (unsigned)cd.y;
    const unsigned long long p1 = a > b ? (a << 16 | b) : (b << 16 | a);
    const unsigned long long p2 = c > d ? (c << 16 | d) : (d << 16 | c);
    return fp_mix64(p1 > p2 ? (p1 << 32 | p2) : (p2 << 32 | p1));
}

__global__ void __launch_bounds__(CLASS_THREADS) quartet_fp_kernel(ClassArgs a, unsigned long long *out) {
    const int ntasks = a.ntasks_dev ? *a.ntasks_dev : a.ntasks;
    if ((int)blockIdx.x >= ntasks) return;
    const int4 t = a.tasks[blockIdx.x];
    const int2 ab = a.b.pair_shell[a.bra_ids[t.x]];
    unsigned long long n = 0, sum = 0, x = 0;
    for (int qi = threadIdx.x; qi < t.z; qi += CLASS_THREADS) {
        const int j = t.y + qi;
        if (!quartet_owned(a, t.x, j)) continue;
        const unsigned long long f = quartet_fp(ab, a.b.pair_shell[a.ket_ids[j]]);
        n++;
        sum += f;
        x ^= f;
    }
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        x ^= __shfl_xor_sync(0xffffffffu, x, o);
    }
    if ((threadIdx.x & 31) == 0 && n) {
        atomicAdd(out, n);
        atomicAdd(out + 1, sum);
        atomicXor(out + 2, x);
    }
}

// ---- launchers -------------------------------------------------------------------
static ClassArgs single_args(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs, int nbf,
                             int tile_rows);

cudaError_t launch_quartet_fp(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs,
                              unsigned long long *out) {
    if (plan.ntasks <= 0) return cudaSuccess;
    const ClassArgs a = single_args(k, ctx, plan, rs, 0, 0);
    quartet_fp_kernel<<<(unsigned)plan.ntasks, CLASS_THREADS, 0, ctx.stream>>>(a, out);
    return cudaGetLastError();
}

cudaError_t launch_class(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs, int precision,
                         int nbf, int tile_rows, int variant) {
    const ClassArgs a = single_args(k, ctx, plan, rs, nbf, tile_rows);
#define LIBERI_CASE(kk, A, B, C, D) \
    case kk: return launch_t<A, B, C, D>(a, precision, variant, ctx.stream);
    switch (k) { LIBERI_CLASSES(LIBERI_CASE) }
#undef LIBERI_CASE
    return cudaErrorInvalidValue;
}

// kernel arguments of one single-molecule class launch over a plan's task list
static ClassArgs single_args(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs, int nbf,
                             int tile_rows) {
    const KernelDesc &kd = KDESC[k];
    ClassArgs a;
    a.b = ctx.basis;
    a.tab = ctx.rys_tab;
    a.tabf = ctx.rys_tabf;
    a.Dm = ctx.D;
    a.Dmf = ctx.Df;
    a.F = ctx.F;
    a.cut = kd.digest_schwarz ? ctx.schwarz_cut : ctx.eri_cut;
    a.thr = kd.asym;
    a.strict = !kd.rys;
    a.tasks = plan.tasks;
    a.ntasks_dev = plan.ntasks_dev;
    a.ntasks = plan.ntasks;
    a.nbf = nbf;
    a.tile_rows = tile_rows;
    a.bra_ids = plan.bra_ids;
    a.ket_ids = plan.ket_ids;
    a.ket_rec = plan.ket_rec;
    a.bra_orig = plan.bra_orig;
    a.ket_orig = plan.ket_orig;
    a.swapped = plan.swapped ? 1 : 0;
    a.rs = rs;
    a.mols = nullptr;
    a.cviews = nullptr;
    a.maxd = ctx.maxd;
    a.prim_cut = ctx.prim_cut;
    a.k_offset = ctx.k_offset;
    return a;
}

cudaError_t launch_class_batch(int k, const LaunchCtx &ctx, const int4 *tasks, int ntasks, int nbf_max,
                               const MolView *d_mols, const ClassView *d_cviews, bool swapped, int precision,
                               const int *ntasks_dev) {
    const KernelDesc &kd = KDESC[k];
    ClassArgs a{};
    a.b = DevBasis{};
    a.tab = ctx.rys_tab;
    a.tabf = ctx.rys_tabf;
    a.Dm = nullptr;
    a.Dmf = nullptr;
    a.F = nullptr;
    a.cut = kd.digest_schwarz ? ctx.schwarz_cut : ctx.eri_cut;
    a.thr = kd.asym;
    a.strict = !kd.rys;
    a.tasks = tasks;
    a.ntasks_dev = ntasks_dev;
    a.ntasks = ntasks;
    a.nbf = nbf_max;
    // F rows are updated with FP64 atomics in L2 (no shared-memory tile), as
    // for single-molecule builds by default
    a.tile_rows = 0;
    a.bra_ids = a.ket_ids = a.bra_orig = a.ket_orig = nullptr;
    a.ket_rec = nullptr;
    a.swapped = swapped ? 1 : 0;
    a.rs = RankSplit{0, 1, 0, 0, 0, 0, 0, 0};
    a.mols = d_mols;
    a.cviews = d_cviews;
    a.maxd = ctx.maxd;
    a.prim_cut = ctx.prim_cut;
    a.k_offset = ctx.k_offset;
#define LIBERI_CASE(kk, A, B, C, D) \
    case kk: return launch_t<A, B, C, D>(a, precision, 0, ctx.stream);
    switch (k) { LIBERI_CLASSES(LIBERI_CASE) }
#undef LIBERI_CASE
    return cudaErrorInvalidValue;
}

__global__ void unpack_kernel(const double *__restrict__ packed, unsigned n, double *__restrict__ sq,
                              float *__restrict__ sqf) {
    const long long total = (long long)n * n;  // n <= 65535: an index fits unsigned 32-bit
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const unsigned i = (unsigned)g, r = i / n, c = i - r * n;
        const double d = packed[tri0(r, c)];
        sq[i] = d;
        if (sqf) sqf[i] = (float)d;
    }
}

// Open-shell builds: sq = ca * A + cb * B as a full n x n matrix (and its float copy)
__global__ void unpack_combo_kernel(const double *__restrict__ pa, const double *__restrict__ pb, double ca,
                                    double cb, unsigned n, double *__restrict__ sq, float *__restrict__ sqf) {
    const long long total = (long long)n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        const unsigned i = (unsigned)g, r = i / n, c = i - r * n;
        const unsigned t = tri0(r, c);
        const double d = ca * pa[t] + cb * pb[t];
        sq[i] = d;
        if (sqf) sqf[i] = (float)d;
    }
}

cudaError_t launch_unpack_combo(const double *pa, const double *pb, double ca, double cb, int n, double *sq,
                                float *sqf, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    const long long want = ((long long)n * n + threads - 1) / threads;
    const int blocks = (int)(want < 148LL * 8 ? want : 148LL * 8);
    unpack_combo_kernel<<<blocks, threads, 0, st>>>(pa, pb, ca, cb, (unsigned)n, sq, sqf);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const double *packed, int n, double *sq, float *sqf, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    const long long want = ((long long)n * n + threads - 1) / threads;
    const int blocks = (int)(want < 148LL * 8 ? want : 148LL * 8);
    unpack_kernel<<<blocks, threads, 0, st>>>(packed, (unsigned)n, sq, sqf);
    return cudaGetLastError();
}

__global__ void zero_fock_kernel(const MolView *mols, int nmol, long long max_ntri) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < (long long)nmol * max_ntri;
         g += stride) {
        const int m = (int)(g / max_ntri);
        const long long i = g - (long long)m * max_ntri;
        const long long n = mols[m].nbf;
        if (i < n * (n + 1) / 2) mols[m].F[i] = 0.0;
    }
}

// per molecule: max|D| (non-negative doubles order as their bits) and D in float
__global__ void batch_prep_kernel(const MolView *mols, int nmol, long long max_nsq, unsigned long long *maxd) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < (long long)nmol * max_nsq;
         g += stride) {
        const int m = (int)(g / max_nsq);
        const unsigned i = (unsigned)(g - (long long)m * max_nsq);
        const unsigned n = (unsigned)mols[m].nbf;
        if (i >= n * n) continue;
        const unsigned r = i / n, c = i - r * n;
        const double d = mols[m].D[tri0(r, c)];
        mols[m].Dsq[i] = d;
        if (mols[m].Df) mols[m].Df[i] = (float)d;
        if (maxd && c <= r) atomicMax(maxd + m, (unsigned long long)__double_as_longlong(fabs(d)));
    }
}

cudaError_t launch_batch_prep(const MolView *d_mols, int nmol, long long max_nsq, unsigned long long *maxd,
                              cudaStream_t st) {
    if (maxd) {
        cudaError_t e = cudaMemsetAsync(maxd, 0, (size_t)nmol * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
    }
    const long long total = (long long)nmol * max_nsq;
    const int threads = 256;
    const long long want = (total + threads - 1) / threads;
    const int blocks = (int)(want < 148LL * 16 ? (want > 0 ? want : 1) : 148LL * 16);
    batch_prep_kernel<<<blocks, threads, 0, st>>>(d_mols, nmol, max_nsq, maxd);
    return cudaGetLastError();
}

cudaError_t launch_zero_fock(const MolView *d_mols, int nmol, long long max_ntri, cudaStream_t st) {
    if (nmol <= 0) return cudaSuccess;
    long long blocks = ((long long)nmol * max_ntri + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    zero_fock_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_mols, nmol, max_ntri);
    return cudaGetLastError();
}

cudaError_t launch_schwarz(int pc, int npairs, int pair_off, const DevBasis &b, const double *tab, double *out,
                           cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    const int threads = 64;
    const unsigned blocks = (unsigned)((npairs + threads - 1) / threads);
    switch (pc) {
        case SS: schwarz_kernel<0, 0><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case SP: schwarz_kernel<1, 0><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case PP: schwarz_kernel<1, 1><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case SD: schwarz_kernel<2, 0><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case PD: schwarz_kernel<2, 1><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        case DD: schwarz_kernel<2, 2><<<blocks, threads, 0, st>>>(b, pair_off, npairs, tab, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_maxabs(const double *x, long long n, unsigned long long *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    long long blocks = (n + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    if (blocks < 1) blocks = 1;
    maxabs_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, n, out);
    return cudaGetLastError();
}

cudaError_t launch_split_tasks(int nitems, const int4 *items, const double *bra_x, const double *ket_x,
                               const unsigned long long *maxd, double fp32_cut, int chunk, int4 *tasks64,
                               int4 *tasks32, int *counts, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counts, 0, 4 * sizeof(int), st);
    if (e != cudaSuccess || nitems <= 0) return e;
    split_tasks_kernel<false><<<(nitems + 255) / 256, 256, 0, st>>>(nitems, items, bra_x, ket_x, nullptr, maxd,
                                                                    fp32_cut, chunk, tasks64, tasks32, counts);
    return cudaGetLastError();
}

cudaError_t launch_split_batch(int nitems, const int4 *items, const ClassView *d_cviews,
                               const unsigned long long *maxd, double fp32_cut, int chunk, int4 *tasks64,
                               int4 *tasks32, int *counts, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(counts, 0, 4 * sizeof(int), st);
    if (e != cudaSuccess || nitems <= 0) return e;
    split_tasks_kernel<true><<<(nitems + 255) / 256, 256, 0, st>>>(nitems, items, nullptr, nullptr, d_cviews, maxd,
                                                                   fp32_cut, chunk, tasks64, tasks32, counts);
    return cudaGetLastError();
}

}  // namespace liberi
