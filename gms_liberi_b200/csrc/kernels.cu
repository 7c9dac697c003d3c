// kernels.cu -- class dispatch, Schwarz generator and mixed-precision split
// kernels of the Fock-build engine; the class kernels themselves are
// instantiated in k_*.cu from quartet.cuh.
#include "quartet.cuh"

namespace liberi {

extern template cudaError_t launch_t<0, 0, 0, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<0, 0, 1, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<0, 0, 1, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 0, 1, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 0, 1, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 1, 1, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<0, 0, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<0, 0, 2, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 0, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 0, 2, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<0, 0, 2, 2>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 0, 2, 2>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<1, 1, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 0, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 2, 1, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 1, 2, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 1, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 1, 1, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 2, 2, 0>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 2, 2, 1>(const ClassArgs &, long long, int, int, cudaStream_t);
extern template cudaError_t launch_t<2, 2, 2, 2>(const ClassArgs &, long long, int, int, cudaStream_t);

// Schwarz table: sqrt(max |(ab|ab)|) per pair of one class
template <int LA, int LB>
__global__ void __launch_bounds__(64) schwarz_kernel(DevBasis b, int pair_off, int npairs,
                                                     const double *tab, double *out) {
    using Q = Quartet<LA, LB, LA, LB, double>;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    int P = pair_off + t;
    double acc[Q::NCART];
    Q::eval(b, P, P, RYS_TMAX, false, tab, acc);
    double m = 0.0;
    for (int ia = 0; ia < Q::NA; ia++)
        for (int ib = 0; ib < Q::NB; ib++) {
            double v = fabs(acc[((ia * Q::NB + ib) * Q::NA + ia) * Q::NB + ib]);
            int n3 = 2 * (cs3(LA, ia) + cs3(LB, ib));
            if (n3 == 2) v *= 3.0; else if (n3 == 4) v *= 9.0;
            m = v > m ? v : m;
        }
    out[t] = sqrt(m);
}

// ---- mixed-precision split --------------------------------------------------------
__global__ void maxabs_kernel(const double *x, long long n, unsigned long long *out) {
    double m = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __double_as_longlong(m));
}

// per bra: split = #kets (of its prefix) with x_bra*x_ket*max|D| >= fp32_cut,
// then exclusive scans of the FP64 and FP32 counts (one CTA per plan)
__global__ void __launch_bounds__(1024) split_kernel(int nbra, const double *bra_x,
                                                     const double *ket_x, const int *ncount,
                                                     const unsigned long long *maxd_bits,
                                                     double fp32_cut, int *split,
                                                     long long *pref64, long long *pref32) {
    __shared__ long long s64[1024], s32[1024];
    const double maxd = __longlong_as_double((long long)*maxd_bits);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per = (nbra + nt - 1) / nt;
    const int i0 = tid * per, i1 = min(nbra, i0 + per);
    long long c64 = 0, c32 = 0;
    for (int i = i0; i < i1; i++) {
        const int n = ncount[i];
        const double xb = bra_x[i];
        int lo = 0, hi = n;  // first position failing the FP64 test
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (xb * ket_x[mid] * maxd >= fp32_cut) lo = mid + 1; else hi = mid;
        }
        split[i] = lo;
        c64 += lo;
        c32 += n - lo;
    }
    s64[tid] = c64;
    s32[tid] = c32;
    __syncthreads();
    for (int off = 1; off < nt; off <<= 1) {
        long long a = tid >= off ? s64[tid - off] : 0, b2 = tid >= off ? s32[tid - off] : 0;
        __syncthreads();
        s64[tid] += a;
        s32[tid] += b2;
        __syncthreads();
    }
    long long r64 = tid > 0 ? s64[tid - 1] : 0, r32 = tid > 0 ? s32[tid - 1] : 0;
    for (int i = i0; i < i1; i++) {
        pref64[i] = r64;
        pref32[i] = r32;
        r64 += split[i];
        r32 += ncount[i] - split[i];
    }
    if (tid == nt - 1) {
        pref64[nbra] = s64[nt - 1];
        pref32[nbra] = s32[nt - 1];
    }
}

// ---- launchers -------------------------------------------------------------------

cudaError_t launch_class(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs,
                         int precision) {
    const KernelDesc &kd = KDESC[k];
    ClassArgs a;
    a.b = ctx.basis;
    a.tab = ctx.rys_tab;
    a.Dm = ctx.D;
    a.F = ctx.F;
    a.cut = kd.digest_schwarz ? ctx.schwarz_cut : ctx.eri_cut;
    a.thr = kd.asym;
    a.strict = !kd.rys;
    a.nbra = plan.nbra;
    a.bra_ids = plan.bra_ids;
    a.ket_ids = plan.ket_ids;
    a.bra_orig = plan.bra_orig;
    a.ket_orig = plan.ket_orig;
    a.pref = plan.pref;
    a.koff = plan.split;
    a.rs = rs;
    const long long w = plan.total;
    switch (k) {
        case 0: return launch_t<0, 0, 0, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 1: return launch_t<0, 0, 1, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 2: return launch_t<0, 0, 1, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 3: return launch_t<1, 0, 1, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 4: return launch_t<1, 0, 1, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 5: return launch_t<1, 1, 1, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 6: return launch_t<0, 0, 2, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 7: return launch_t<0, 0, 2, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 8: return launch_t<1, 0, 2, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 9: return launch_t<1, 0, 2, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 10: return launch_t<0, 0, 2, 2>(a, w, precision, ctx.num_sms, ctx.stream);
        case 11: return launch_t<1, 0, 2, 2>(a, w, precision, ctx.num_sms, ctx.stream);
        case 12: return launch_t<1, 1, 2, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 13: return launch_t<2, 0, 2, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 14: return launch_t<2, 2, 1, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 15: return launch_t<2, 1, 2, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 16: return launch_t<2, 1, 2, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 17: return launch_t<2, 1, 1, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 18: return launch_t<2, 2, 2, 0>(a, w, precision, ctx.num_sms, ctx.stream);
        case 19: return launch_t<2, 2, 2, 1>(a, w, precision, ctx.num_sms, ctx.stream);
        case 20: return launch_t<2, 2, 2, 2>(a, w, precision, ctx.num_sms, ctx.stream);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_schwarz(int pc, int npairs, int pair_off, const DevBasis &b,
                           const double *tab, double *out, cudaStream_t st) {
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

cudaError_t launch_split(int nbra, const double *bra_x, const double *ket_x, const int *ncount,
                         const unsigned long long *maxd, double fp32_cut, int *split,
                         long long *pref64, long long *pref32, cudaStream_t st) {
    if (nbra <= 0) return cudaSuccess;
    split_kernel<<<1, 1024, 0, st>>>(nbra, bra_x, ket_x, ncount, maxd, fp32_cut, split, pref64,
                                     pref32);
    return cudaGetLastError();
}


}  // namespace liberi
