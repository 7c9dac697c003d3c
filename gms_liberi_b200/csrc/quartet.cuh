// quartet.cuh -- sm_100a device code of the quartet classes (included by the
// per-class translation units k_*.cu and by kernels.cu).
//
// One templated kernel per reference quartet class intABCD
// (src/rhf/rot_axis/int*.F90, driver order src/liberi_driver.F90:69-102).
//
// Work unit: a CTA owns one "row" shell pair P = (A, B) and a chunk of its
// surviving ket pairs Q = (C, D) (the kets of a bra form a prefix of the
// Schwarz-sorted ket list).  Each thread evaluates whole quartets:
//   1. loop over kept primitive pairs (ket outer, bra inner, as the reference
//      does, e.g. int0001.F90:220-287), evaluate Rys roots and weights from
//      the piecewise tables, build 2D integrals with the vertical and
//      horizontal recurrences in registers and contract the Cartesian block;
//      large classes run the primitive loop in register-bounded passes over
//      the components of shell A;
//   2. digest with the reference's DIRFCK rules (unique components for
//      identical shells, 0.5 factors, skip |v| < cut, the six updates of
//      int0000.F90:241-311 / int2222_rysgen.F90:11176-11338), pre-reduced in
//      registers per quartet:
//        K updates into rows A and B of F -> shared-memory tile of the CTA
//        J update of the row pair (A,B)   -> summed over the warp (shuffles),
//                                            one tile update per warp
//        J update of the ket pair (C,D)   -> FP64 global atomics
//      and the tile is flushed to F with FP64 atomics when the CTA ends.
// The FP32 instantiation evaluates step 1 entirely in single precision (pair
// data rounded once from FP64, Rys roots and weights from single-precision
// tables, recurrences and contraction) for the quartets whose Schwarz bound
// times max|D| falls below the mixed-precision cut; step 2 always digests in
// FP64.
#pragma once
#include <cstdio>
#include <type_traits>

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
// 256-bit read-only loads (sm_100): a function's coefficients are 32-byte
// aligned in both tables (offsets are multiples of 64 bytes from a 256-byte
// aligned base), so one lane fetches four doubles (or eight floats) per load.
__device__ __forceinline__ void ldg_v4f64(const double *p, double &a, double &b, double &c, double &d) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
        : "l"((unsigned long long)__cvta_generic_to_global(p)));
}
__device__ __forceinline__ double4 ldg_double4(const double4 *p) {
    double4 v;
    ldg_v4f64(reinterpret_cast<const double *>(p), v.x, v.y, v.z, v.w);
    return v;
}
__device__ __forceinline__ void ldg_v8f32(const float *p, float4 &lo, float4 &hi) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z), "=f"(hi.w)
        : "l"((unsigned long long)__cvta_generic_to_global(p)));
}
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
    const double t4 = T * (double)RYS_PER_UNIT;
    const int k = (int)t4;
    const double x = 2.0 * (t4 - (double)k) - 1.0;
    const double *base = tab + rys_table_off(N) + (size_t)k * (2 * N * RYS_NCOEF);
    // two 256-bit loads per function; Estrin evaluation, dependency depth 3
    const double x2 = x * x, x4 = x2 * x2;
#pragma unroll
    for (int f = 0; f < 2 * N; f++) {
        double c0, c1, c2, c3, c4, c5, c6, c7;
        ldg_v4f64(base + f * RYS_NCOEF, c0, c1, c2, c3);
        ldg_v4f64(base + f * RYS_NCOEF + 4, c4, c5, c6, c7);
        const double a0 = fma(c1, x, c0), a1 = fma(c3, x, c2);
        const double a2 = fma(c5, x, c4), a3 = fma(c7, x, c6);
        const double b0 = fma(a1, x2, a0), b1 = fma(a3, x2, a2);
        const double v = fma(b1, x4, b0);
        if (f < N) u[f] = v; else w[f - N] = v;
    }
}

// Table rows staged in shared memory: the classes with the large-T form from
// T = 25 (the reference's t_max) need intervals 0..100 only; a CTA copies its
// class's rows at start, each row padded by 16 bytes (stride 16N+2 doubles)
// so that lanes reading different rows spread over the banks, and reads them
// with 128-bit shared loads.  Measured per class on C60 (FP64): (ss|pp)
// 6.17 -> 5.91 ms, (sp|sp) 14.21 -> 14.11, (ss|dd) 0.353 -> 0.336; slower in
// the other classes ((ss|ss) 2.78 -> 3.14, (pp|pp) 9.63 -> 10.48, (ss|sd)
// 1.91 -> 2.22 ms): the copy and the random-row bank conflicts cost more than
// the L1 misses they save, so only those three stage their rows.
constexpr int STAB_NINT = 25 * RYS_PER_UNIT + 1;
__host__ __device__ constexpr int stab_stride(int n) { return 16 * n + 2; }
template <int N>
__device__ __forceinline__ void rys_eval_staged(double T, double thr, bool strict, const double *__restrict__ tab,
                                                const double *stab, double *u, double *w) {
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
    const double t4 = T * (double)RYS_PER_UNIT;
    const int k = (int)t4;
    const double x = 2.0 * (t4 - (double)k) - 1.0;
    const double *base = stab + k * stab_stride(N);
    const double x2 = x * x, x4 = x2 * x2;
#pragma unroll
    for (int f = 0; f < 2 * N; f++) {
        const double2 q0 = *reinterpret_cast<const double2 *>(base + f * RYS_NCOEF);
        const double2 q1 = *reinterpret_cast<const double2 *>(base + f * RYS_NCOEF + 2);
        const double2 q2 = *reinterpret_cast<const double2 *>(base + f * RYS_NCOEF + 4);
        const double2 q3 = *reinterpret_cast<const double2 *>(base + f * RYS_NCOEF + 6);
        const double a0 = fma(q0.y, x, q0.x), a1 = fma(q1.y, x, q1.x);
        const double a2 = fma(q2.y, x, q2.x), a3 = fma(q3.y, x, q3.x);
        const double b0 = fma(a1, x2, a0), b1 = fma(a3, x2, a2);
        const double v = fma(b1, x4, b0);
        if (f < N) u[f] = v; else w[f - N] = v;
    }
}
// the classes that stage their rows (FP64 (ss|pp), (sp|sp), (ss|dd))
template <int LA, int LB, int LC, int LD, typename R>
constexpr bool stab_class() {
    constexpr int key = LA * 1000 + LB * 100 + LC * 10 + LD;
    return std::is_same<R, double>::value && (key == 1100 || key == 1010 || key == 2200);
}
template <int LA, int LB, int LC, int LD, typename R>
constexpr size_t stab_bytes() {
    return stab_class<LA, LB, LC, LD, R>() ? (size_t)STAB_NINT * stab_stride((LA + LB + LC + LD) / 2 + 1) * 8 : 0;
}

// FP32 tier: width-1/8 intervals, degree 3 (two functions per 256-bit load);
// the large-T limit as in FP64.
template <int N>
__device__ __forceinline__ void rys_eval(float T, float thr, bool strict, const float *__restrict__ tab, float *u,
                                         float *w) {
    bool asym = strict ? (T > thr) : (T >= thr);
    if (asym) {
        const float sq = rsqrtf(T), it = sq * sq;
        const float *hr = tab + rysf_herm_off(N);
#pragma unroll
        for (int i = 0; i < N; i++) {
            u[i] = __ldg(hr + i) * it;
            w[i] = __ldg(hr + MAXROOT + i) * sq;
        }
        return;
    }
    const float t8 = T * (float)RYSF_PER_UNIT;
    const int k = (int)t8;
    const float x = 2.0f * (t8 - (float)k) - 1.0f;
    const float *base = tab + rysf_table_off(N) + (size_t)k * (2 * N * RYSF_NCOEF);
    const float x2 = x * x;
#pragma unroll
    for (int f = 0; f < 2 * N; f += 2) {  // two functions per 256-bit load
        float4 c0, c1;
        ldg_v8f32(base + f * RYSF_NCOEF, c0, c1);
        const float v0 = fmaf(fmaf(c0.w, x, c0.z), x2, fmaf(c0.y, x, c0.x));
        const float v1 = fmaf(fmaf(c1.w, x, c1.z), x2, fmaf(c1.y, x, c1.x));
        if (f < N) u[f] = v0; else w[f - N] = v0;
        if (f + 1 < N) u[f + 1] = v1; else w[f + 1 - N] = v1;
    }
}

// ---- two Rys roots in one packed FP32 pair (FP32 tier) ------------------------
// F2 holds one quantity for two roots of a primitive quartet; its arithmetic
// is the paired single-precision instructions of sm_100 (__fmul2_rn,
// __fadd2_rn, __ffma2_rn), so the recurrences and transfers of two roots
// issue as one.  A product is kept unrounded (F2P) until it meets an addition,
// which then becomes one fused multiply-add, as the compiler contracts the
// scalar code.
struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ explicit F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
};
struct F2P {
    float2 a, b;
    __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a, b)); }
};
__device__ __forceinline__ F2P operator*(F2 x, F2 y) { return F2P{x.v, y.v}; }
__device__ __forceinline__ F2P operator*(F2P x, F2 y) { return F2P{__fmul2_rn(x.a, x.b), y.v}; }
__device__ __forceinline__ F2 operator+(F2 x, F2 y) { return F2(__fadd2_rn(x.v, y.v)); }
__device__ __forceinline__ F2 operator+(F2 x, F2P y) { return F2(__ffma2_rn(y.a, y.b, x.v)); }
__device__ __forceinline__ F2 operator+(F2P x, F2 y) { return F2(__ffma2_rn(x.a, x.b, y.v)); }
__device__ __forceinline__ F2 operator+(F2P x, F2P y) { return F2(__ffma2_rn(x.a, x.b, __fmul2_rn(y.a, y.b))); }
__device__ __forceinline__ F2 &operator+=(F2 &x, F2P y) { x = F2(__ffma2_rn(y.a, y.b, x.v)); return x; }
__device__ __forceinline__ F2 &operator+=(F2 &x, F2 y) { x = F2(__fadd2_rn(x.v, y.v)); return x; }
// FP32 classes that run their roots in pairs.  Measured per class on C60
// (mixed builds, every FP32 class with two or more roots paired): (pd|pd)
// 3.05 -> 2.91 ms at cut 1e-2 and 3.36 -> 3.22 ms at 1e-5; the others lost or
// did not change ((pd|pp) 6.17 -> 6.71, (sp|pd) 5.16 -> 5.47, all paired:
// 49.3 -> 50.7 ms at cut 1e-2), the packing moves costing what the paired
// instructions save.
constexpr bool pair_roots_class(int key) { return key == 2121; }

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

// ---- (e0|c0) intermediates: contraction before the bra transfer ---------------
// Cartesian components of angular momentum l <= 4 in a fixed order: the
// engine's order for l <= 2 (x,y,z; xx,yy,zz,xy,xz,yz), otherwise x exponent
// descending, then y descending.  Switch tables (not loops), so that the
// compiler folds them at once inside the unrolled contraction and transfer.
__host__ __device__ constexpr int cart_x(int l, int i) {
    if (l <= 2) return cxp(l, i);
    switch (l * 16 + i) {
        case 0: return 0;
        case 16: return 1;
        case 17: return 0;
        case 18: return 0;
        case 32: return 2;
        case 33: return 0;
        case 34: return 0;
        case 35: return 1;
        case 36: return 1;
        case 37: return 0;
        case 48: return 3;
        case 49: return 2;
        case 50: return 2;
        case 51: return 1;
        case 52: return 1;
        case 53: return 1;
        case 54: return 0;
        case 55: return 0;
        case 56: return 0;
        case 57: return 0;
        case 64: return 4;
        case 65: return 3;
        case 66: return 3;
        case 67: return 2;
        case 68: return 2;
        case 69: return 2;
        case 70: return 1;
        case 71: return 1;
        case 72: return 1;
        case 73: return 1;
        case 74: return 0;
        case 75: return 0;
        case 76: return 0;
        case 77: return 0;
        case 78: return 0;
        default: return 0;
    }
}
__host__ __device__ constexpr int cart_y(int l, int i) {
    if (l <= 2) return cyp(l, i);
    switch (l * 16 + i) {
        case 0: return 0;
        case 16: return 0;
        case 17: return 1;
        case 18: return 0;
        case 32: return 0;
        case 33: return 2;
        case 34: return 0;
        case 35: return 1;
        case 36: return 0;
        case 37: return 1;
        case 48: return 0;
        case 49: return 1;
        case 50: return 0;
        case 51: return 2;
        case 52: return 1;
        case 53: return 0;
        case 54: return 3;
        case 55: return 2;
        case 56: return 1;
        case 57: return 0;
        case 64: return 0;
        case 65: return 1;
        case 66: return 0;
        case 67: return 2;
        case 68: return 1;
        case 69: return 0;
        case 70: return 3;
        case 71: return 2;
        case 72: return 1;
        case 73: return 0;
        case 74: return 4;
        case 75: return 3;
        case 76: return 2;
        case 77: return 1;
        case 78: return 0;
        default: return 0;
    }
}
__host__ __device__ constexpr int cart_z(int l, int i) { return l - cart_x(l, i) - cart_y(l, i); }
// index of the component (x, y, l-x-y) within angular momentum l
__host__ __device__ constexpr int cart_pos(int l, int x, int y) {
    if (l == 0) return 0;
    if (l == 1) return x == 1 ? 0 : (y == 1 ? 1 : 2);
    if (l == 2) return x == 2 ? 0 : (y == 2 ? 1 : (x + y == 0 ? 2 : (x == 1 && y == 1 ? 3 : (x == 1 ? 4 : 5))));
    switch (l * 100 + x * 10 + y) {
        case 0: return 0;
        case 110: return 0;
        case 101: return 1;
        case 100: return 2;
        case 220: return 0;
        case 202: return 1;
        case 200: return 2;
        case 211: return 3;
        case 210: return 4;
        case 201: return 5;
        case 330: return 0;
        case 321: return 1;
        case 320: return 2;
        case 312: return 3;
        case 311: return 4;
        case 310: return 5;
        case 303: return 6;
        case 302: return 7;
        case 301: return 8;
        case 300: return 9;
        case 440: return 0;
        case 431: return 1;
        case 430: return 2;
        case 422: return 3;
        case 421: return 4;
        case 420: return 5;
        case 413: return 6;
        case 412: return 7;
        case 411: return 8;
        case 410: return 9;
        case 404: return 10;
        case 403: return 11;
        case 402: return 12;
        case 401: return 13;
        case 400: return 14;
        default: return 0;
    }
}
// Cartesian functions with angular momentum LA..LA+LB, in order of l
// (closed forms and ternaries, not recursion: the compiler must fold every
// index below before it places the arrays they address)
__host__ __device__ constexpr int ncart_upto(int n) { return n < 0 ? 0 : (n + 1) * (n + 2) * (n + 3) / 6; }
__host__ __device__ constexpr int nrange(int l0, int l1) { return l1 < l0 ? 0 : ncart_upto(l1) - ncart_upto(l0 - 1); }
__host__ __device__ constexpr int range_pos(int l0, int x, int y, int z) {
    return nrange(l0, x + y + z - 1) + cart_pos(x + y + z, x, y);
}
__host__ __device__ constexpr int binom2(int n, int k) { return (k == 0 || k == n) ? 1 : n; }  // n <= 2

// Classes evaluated as (e0|c0) intermediates: single-pass classes with a
// p or d second bra shell and an s second ket shell.  The VRR blocks of each
// root are contracted straight into (e0|c0), e over the Cartesian functions
// of angular momentum L_A..L_A+L_B (the transfer to (ab|c0) needs only A-B,
// the same for every primitive), and the bra transfer runs once per quartet
// instead of once per root: fewer FP64 operations per root and no per-root
// transfer block held in registers.
template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr bool hgp_class(int npass) {
    return npass == 1 && LB > 0 && LD == 0;
}

// angular momentum and component of the e-th function of the range starting at l0
__host__ __device__ constexpr int range_l(int l0, int e) {
    return e < nrange(l0, l0) ? l0
         : e < nrange(l0, l0 + 1) ? l0 + 1
         : e < nrange(l0, l0 + 2) ? l0 + 2
         : e < nrange(l0, l0 + 3) ? l0 + 3
                                  : l0 + 4;
}
__host__ __device__ constexpr int range_i(int l0, int e) { return e - nrange(l0, range_l(l0, e) - 1); }

// Loop bounds below are compile-time constants (the flat range index e, and
// transfer exponents up to L_B with guards): a bound that depends on an outer
// loop index is not fully unrolled, and the arrays it indexes then live in
// local memory.
template <int LA, int LB, int LC, typename R>
__device__ __forceinline__ void contract_hgp(const R (&gx)[LA + LB + 1][LC + 1], const R (&gy)[LA + LB + 1][LC + 1],
                                             const R (&gz)[LA + LB + 1][LC + 1],
                                             R (&acc)[nrange(LA, LA + LB)][ncart(LC)]) {
#pragma unroll
    for (int e = 0; e < nrange(LA, LA + LB); e++) {
        const int le = range_l(LA, e), ie = range_i(LA, e);
#pragma unroll
        for (int ic = 0; ic < ncart(LC); ic++)
            acc[e][ic] = fma(gx[cart_x(le, ie)][cxp(LC, ic)] * gy[cart_y(le, ie)][cyp(LC, ic)],
                             gz[cart_z(le, ie)][czp(LC, ic)], acc[e][ic]);
    }
}

// (a b|c0) for A component ia (a compile-time index) from the contracted
// (e0|c0): (a b| = sum_{t <= b} prod_i binom(b_i, t_i) (A-B)_i^(b_i - t_i) (a+t 0|
template <int LA, int LB, int LC, typename R>
__device__ __forceinline__ void bra_transfer(const R (&acc)[nrange(LA, LA + LB)][ncart(LC)], int ia, R abx, R aby,
                                             R abz, R (&sl)[ncart(LB)][ncart(LC)][1]) {
    const int ax = cxp(LA, ia), ay = cyp(LA, ia), az = czp(LA, ia);
    const R px[3] = {R(1), abx, abx * abx}, py[3] = {R(1), aby, aby * aby}, pz[3] = {R(1), abz, abz * abz};
#pragma unroll
    for (int ib = 0; ib < ncart(LB); ib++) {
        const int bx = cxp(LB, ib), by = cyp(LB, ib), bz = czp(LB, ib);
#pragma unroll
        for (int ic = 0; ic < ncart(LC); ic++) {
            R v = R(0);
#pragma unroll
            for (int tx = 0; tx <= LB; tx++)
#pragma unroll
                for (int ty = 0; ty <= LB; ty++)
#pragma unroll
                    for (int tz = 0; tz <= LB; tz++) {
                        if (tx > bx || ty > by || tz > bz) continue;
                        const R c = R(binom2(bx, tx) * binom2(by, ty) * binom2(bz, tz)) * px[bx - tx] * py[by - ty] *
                                    pz[bz - tz];
                        v = fma(c, acc[range_pos(LA, ax + tx, ay + ty, az + tz)][ic], v);
                    }
            sl[ib][ic][0] = v;
        }
    }
}

// ---- contracted Cartesian block of one shell quartet -------------------------
// Component tables as runtime values (used to select one A component).
__device__ __forceinline__ int cx_rt(int l, int c) { return l == 0 ? 0 : (l == 1 ? (c == 0) : (c == 0 ? 2 : ((c == 3 || c == 4) ? 1 : 0))); }
__device__ __forceinline__ int cy_rt(int l, int c) { return l == 0 ? 0 : (l == 1 ? (c == 1) : (c == 1 ? 2 : ((c == 3 || c == 5) ? 1 : 0))); }
__device__ __forceinline__ int cz_rt(int l, int c) { return l == 0 ? 0 : (l == 1 ? (c == 2) : (c == 2 ? 2 : ((c == 4 || c == 5) ? 1 : 0))); }

// horizontal transfer for one runtime A exponent ea: s[b][c][d] = I[ea][b][c][d]
// from the VRR block g[e][f] (rows ea..ea+LB are selected first)
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void hrr_slice(const R (&g)[LA + LB + 1][LC + LD + 1], int ea, R ab, R cd,
                                          R (&s)[LB + 1][LC + 1][LD + 1]) {
    constexpr int LCD = LC + LD;
    R h[LB + 1][LB + 1][LCD + 1];  // h[t][b][f] = I(ea + t, b) before the ket transfer
#pragma unroll
    for (int t = 0; t <= LB; t++)
#pragma unroll
        for (int f = 0; f <= LCD; f++) {
            R v = g[t][f];
#pragma unroll
            for (int x = 1; x <= LA; x++) v = (ea == x) ? g[x + t][f] : v;
            h[t][0][f] = v;
        }
#pragma unroll
    for (int b = 1; b <= LB; b++)
#pragma unroll
        for (int t = 0; t <= LB - b; t++)
#pragma unroll
            for (int f = 0; f <= LCD; f++) h[t][b][f] = h[t + 1][b - 1][f] + ab * h[t][b - 1][f];
#pragma unroll
    for (int b = 0; b <= LB; b++) {
        R k2[LCD + 1][LD + 1];
#pragma unroll
        for (int f = 0; f <= LCD; f++) k2[f][0] = h[0][b][f];
#pragma unroll
        for (int d = 1; d <= LD; d++)
#pragma unroll
            for (int c = 0; c <= LCD - d; c++) k2[c][d] = k2[c + 1][d - 1] + cd * k2[c][d - 1];
#pragma unroll
        for (int c = 0; c <= LC; c++)
#pragma unroll
            for (int d = 0; d <= LD; d++) s[b][c][d] = k2[c][d];
    }
}

// One root's contribution: horizontal transfer of the three 2D blocks and
// accumulation of the contracted Cartesian block (all A components of the
// pass at compile-time indices when the pass covers all of A).
template <int LA, int LB, int LC, int LD, typename R, int NMU>
__device__ __forceinline__ void contract_root(const R (&gx)[LA + LB + 1][LC + LD + 1],
                                              const R (&gy)[LA + LB + 1][LC + LD + 1],
                                              const R (&gz)[LA + LB + 1][LC + LD + 1], R abx, R aby, R abz,
                                              R cdx, R cdy, R cdz, const int (&ex)[NMU], const int (&ey)[NMU],
                                              const int (&ez)[NMU], R (&acc)[NMU][ncart(LB)][ncart(LC)][ncart(LD)]) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr bool FULL = (NMU == NA);
    if constexpr (FULL) {
        R ix[LA + 1][LB + 1][LC + 1][LD + 1], iy[LA + 1][LB + 1][LC + 1][LD + 1],
            iz[LA + 1][LB + 1][LC + 1][LD + 1];
        hrr<LA, LB, LC, LD, R>(gx, abx, cdx, ix);
        hrr<LA, LB, LC, LD, R>(gy, aby, cdy, iy);
        hrr<LA, LB, LC, LD, R>(gz, abz, cdz, iz);
#pragma unroll
        for (int m = 0; m < NMU; m++)
#pragma unroll
            for (int ib = 0; ib < NB; ib++)
#pragma unroll
                for (int ic = 0; ic < NC; ic++)
#pragma unroll
                    for (int id = 0; id < ND; id++)
                        acc[m][ib][ic][id] += ix[cxp(LA, m)][cxp(LB, ib)][cxp(LC, ic)][cxp(LD, id)] *
                                              iy[cyp(LA, m)][cyp(LB, ib)][cyp(LC, ic)][cyp(LD, id)] *
                                              iz[czp(LA, m)][czp(LB, ib)][czp(LC, ic)][czp(LD, id)];
    } else {
#pragma unroll
        for (int m = 0; m < NMU; m++) {
            R sx[LB + 1][LC + 1][LD + 1], sy[LB + 1][LC + 1][LD + 1], sz[LB + 1][LC + 1][LD + 1];
            hrr_slice<LA, LB, LC, LD, R>(gx, ex[m], abx, cdx, sx);
            hrr_slice<LA, LB, LC, LD, R>(gy, ey[m], aby, cdy, sy);
            hrr_slice<LA, LB, LC, LD, R>(gz, ez[m], abz, cdz, sz);
#pragma unroll
            for (int ib = 0; ib < NB; ib++)
#pragma unroll
                for (int ic = 0; ic < NC; ic++)
#pragma unroll
                    for (int id = 0; id < ND; id++)
                        acc[m][ib][ic][id] += sx[cxp(LB, ib)][cxp(LC, ic)][cxp(LD, id)] *
                                              sy[cyp(LB, ib)][cyp(LC, ic)][cyp(LD, id)] *
                                              sz[czp(LB, ib)][czp(LC, ic)][czp(LD, id)];
        }
    }
}

// contract_root for a pair of roots (FP32 tier): the transfers run on the
// packed pair, each integral adds its two roots' products to the scalar
// accumulator (one paired multiply and two fused multiply-adds)
__device__ __forceinline__ float acc_pair(F2 x, F2 y, F2 z, float acc) {
    const float2 t = __fmul2_rn(x.v, y.v);
    return fmaf(t.y, z.v.y, fmaf(t.x, z.v.x, acc));
}
template <int LA, int LB, int LC, int LD, int NMU>
__device__ __forceinline__ void contract_root_pair(const F2 (&gx)[LA + LB + 1][LC + LD + 1],
                                                   const F2 (&gy)[LA + LB + 1][LC + LD + 1],
                                                   const F2 (&gz)[LA + LB + 1][LC + LD + 1], F2 abx, F2 aby, F2 abz,
                                                   F2 cdx, F2 cdy, F2 cdz, const int (&ex)[NMU], const int (&ey)[NMU],
                                                   const int (&ez)[NMU],
                                                   float (&acc)[NMU][ncart(LB)][ncart(LC)][ncart(LD)]) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr bool FULL = (NMU == NA);
    if constexpr (FULL) {
        F2 ix[LA + 1][LB + 1][LC + 1][LD + 1], iy[LA + 1][LB + 1][LC + 1][LD + 1],
            iz[LA + 1][LB + 1][LC + 1][LD + 1];
        hrr<LA, LB, LC, LD, F2>(gx, abx, cdx, ix);
        hrr<LA, LB, LC, LD, F2>(gy, aby, cdy, iy);
        hrr<LA, LB, LC, LD, F2>(gz, abz, cdz, iz);
#pragma unroll
        for (int m = 0; m < NMU; m++)
#pragma unroll
            for (int ib = 0; ib < NB; ib++)
#pragma unroll
                for (int ic = 0; ic < NC; ic++)
#pragma unroll
                    for (int id = 0; id < ND; id++)
                        acc[m][ib][ic][id] = acc_pair(ix[cxp(LA, m)][cxp(LB, ib)][cxp(LC, ic)][cxp(LD, id)],
                                                      iy[cyp(LA, m)][cyp(LB, ib)][cyp(LC, ic)][cyp(LD, id)],
                                                      iz[czp(LA, m)][czp(LB, ib)][czp(LC, ic)][czp(LD, id)],
                                                      acc[m][ib][ic][id]);
    } else {
#pragma unroll
        for (int m = 0; m < NMU; m++) {
            F2 sx[LB + 1][LC + 1][LD + 1], sy[LB + 1][LC + 1][LD + 1], sz[LB + 1][LC + 1][LD + 1];
            hrr_slice<LA, LB, LC, LD, F2>(gx, ex[m], abx, cdx, sx);
            hrr_slice<LA, LB, LC, LD, F2>(gy, ey[m], aby, cdy, sy);
            hrr_slice<LA, LB, LC, LD, F2>(gz, ez[m], abz, cdz, sz);
#pragma unroll
            for (int ib = 0; ib < NB; ib++)
#pragma unroll
                for (int ic = 0; ic < NC; ic++)
#pragma unroll
                    for (int id = 0; id < ND; id++)
                        acc[m][ib][ic][id] = acc_pair(sx[cxp(LB, ib)][cxp(LC, ic)][cxp(LD, id)],
                                                      sy[cyp(LB, ib)][cyp(LC, ic)][cyp(LD, id)],
                                                      sz[czp(LB, ib)][czp(LC, ic)][czp(LD, id)], acc[m][ib][ic][id]);
        }
    }
}
template <int LA, int LB, int LC>
__device__ __forceinline__ void contract_hgp_pair(const F2 (&gx)[LA + LB + 1][LC + 1], const F2 (&gy)[LA + LB + 1][LC + 1],
                                                  const F2 (&gz)[LA + LB + 1][LC + 1],
                                                  float (&acc)[nrange(LA, LA + LB)][ncart(LC)]) {
#pragma unroll
    for (int e = 0; e < nrange(LA, LA + LB); e++) {
        const int le = range_l(LA, e), ie = range_i(LA, e);
#pragma unroll
        for (int ic = 0; ic < ncart(LC); ic++)
            acc[e][ic] = acc_pair(gx[cart_x(le, ie)][cxp(LC, ic)], gy[cart_y(le, ie)][cyp(LC, ic)],
                                  gz[cart_z(le, ie)][czp(LC, ic)], acc[e][ic]);
    }
}

// acc[m][ib][ic][id] for A components ia = mu0 + m (m < NMU, ia < NA), all of
// B, C, D.  A single pass (NMU == NA) uses compile-time component indices; a
// multi-pass class selects the A exponent at run time, so one copy of the
// primitive loop serves every pass and the root loop is not unrolled.
// HGP: acc is the (e0|c0) block of contract_hgp (L_D = 0, one pass), else the
// (ab|cd) block of NMU A components.
template <int LA, int LB, int LC, int LD, typename R, int NMU, bool HGP, typename ACC>
__device__ __forceinline__ void eval_block(const DevBasis &b, int p0, int np, int q0, int nq,
                                           const double4 &A, const double4 &C, R abx, R aby, R abz,
                                           R cdx, R cdy, R cdz, double thr, bool strict,
                                           const double *__restrict__ tab, const float *__restrict__ tabf,
                                           int mu0, ACC &acc, R *cache_u, R *cache_w, int cache,
                                           float pthr = 0.f, float bpmax = 0.f, const double *stab = nullptr) {
    constexpr int NA = ncart(LA);
    constexpr int LAB = LA + LB, LCD = LC + LD;
    constexpr int NR = (LAB + LCD) / 2 + 1;
    constexpr bool FULL = (NMU == NA);
    static_assert(!HGP || (LD == 0 && FULL), "(e0|c0) contraction: one pass, s second ket shell");
    int ex[NMU], ey[NMU], ez[NMU];
#pragma unroll
    for (int m = 0; m < NMU; m++) {
        const int ia = mu0 + m < NA ? mu0 + m : NA - 1;
        ex[m] = cx_rt(LA, ia);
        ey[m] = cy_rt(LA, ia);
        ez[m] = cz_rt(LA, ia);
    }
    if constexpr (HGP) {
#pragma unroll
        for (int e = 0; e < nrange(LA, LA + LB); e++)
#pragma unroll
            for (int ic = 0; ic < ncart(LC); ic++) acc[e][ic] = R(0);
    } else {
#pragma unroll
        for (int m = 0; m < NMU; m++)
#pragma unroll
            for (int ib = 0; ib < ncart(LB); ib++)
#pragma unroll
                for (int ic = 0; ic < ncart(LC); ic++)
#pragma unroll
                    for (int id = 0; id < ncart(LD); id++) acc[m][ib][ic][id] = R(0);
    }
    int slot = 0;  // primitive quartet index within the shell quartet (root cache)
    if constexpr (std::is_same<R, double>::value) {
        for (int kq = q0; kq < q0 + nq; kq++) {
            const double4 Qp = ldg_double4(b.prim_P + kq);
            const double2 Qx = b.prim_X[kq];
            const double q = Qp.w, hq = Qx.y;
            for (int kp = p0; kp < p0 + np; kp++) {
                const double4 Pp = ldg_double4(b.prim_P + kp);
                const double2 Px = b.prim_X[kp];
                const double p = Pp.w, hp = Px.y;
                const double pqx = Pp.x - Qp.x, pqy = Pp.y - Qp.y, pqz = Pp.z - Qp.z;
                double u[NR], w[NR];  // u_i / (p+q) and w_i times the pair prefactors
                if (cache == 2) {
#pragma unroll
                    for (int i = 0; i < NR; i++) {
                        u[i] = cache_u[slot * NR + i];
                        w[i] = cache_w[slot * NR + i];
                    }
                } else {
                    const double rs = rsqrt(p + q);
                    const double ipq = rs * rs;
                    const double T = p * q * ipq * (pqx * pqx + pqy * pqy + pqz * pqz);
                    if (stab_class<LA, LB, LC, LD, R>() && stab != nullptr)
                        rys_eval_staged<NR>(T, thr, strict, tab, stab, u, w);
                    else
                        rys_eval<NR>(T, thr, strict, tab, u, w);
                    const double pref = Px.x * Qx.x * rs;
#pragma unroll
                    for (int i = 0; i < NR; i++) {
                        u[i] *= ipq;
                        w[i] *= pref;
                        if (cache == 1) {
                            cache_u[slot * NR + i] = u[i];
                            cache_w[slot * NR + i] = w[i];
                        }
                    }
                }
                slot++;
#pragma unroll(FULL ? NR : 1)
                for (int r = 0; r < NR; r++) {
                    const double ui = u[0], wr = w[0];
#pragma unroll
                    for (int i = 0; i + 1 < NR; i++) {  // rotate the next root to the front
                        u[i] = u[i + 1];
                        w[i] = w[i + 1];
                    }
                    const double fq = q * ui, fp = p * ui;
                    const R b00 = R(0.5 * ui);
                    const R b10 = R(hp * (1.0 - fq));
                    const R b01 = R(hq * (1.0 - fp));
                    R gx[LAB + 1][LCD + 1], gy[LAB + 1][LCD + 1], gz[LAB + 1][LCD + 1];
                    vrr<LAB, LCD, R>(gx, R((Pp.x - A.x) - fq * pqx), R((Qp.x - C.x) + fp * pqx), b10, b01, b00, R(1));
                    vrr<LAB, LCD, R>(gy, R((Pp.y - A.y) - fq * pqy), R((Qp.y - C.y) + fp * pqy), b10, b01, b00, R(1));
                    vrr<LAB, LCD, R>(gz, R((Pp.z - A.z) - fq * pqz), R((Qp.z - C.z) + fp * pqz), b10, b01, b00,
                                     R(wr));
                    if constexpr (HGP) contract_hgp<LA, LB, LC, R>(gx, gy, gz, acc);
                    else contract_root<LA, LB, LC, LD, R, NMU>(gx, gy, gz, abx, aby, abz, cdx, cdy, cdz, ex, ey, ez, acc);
                }
            }
        }
    } else {
        // FP32 tier: pair data, roots and recurrences in single precision
        const float *__restrict__ PAf = reinterpret_cast<const float *>(b.prim_PAf);
        const float thrf = (float)thr;
        // Primitive screening of the FP32 tier: a primitive quartet whose
        // Schwarz bound bp*bq is below pthr (fp32_prim * fp32_cut / max|D|,
        // far below the rounding error of this tier's quartets) is skipped.
        // Every pair's primitives are stored by decreasing bound, so both
        // loops end at the first primitive below the cut.
        for (int kq = q0; kq < q0 + nq; kq++) {
            const float bq = pthr > 0.f ? __ldg(b.prim_bound + kq) : 1.f;
            if (bq * bpmax < pthr) break;
            float4 Qp, Qa;
            ldg_v8f32(PAf + 8 * (size_t)kq, Qp, Qa);
            const float q = Qp.w, hq = __fdividef(0.5f, q);
            for (int kp = p0; kp < p0 + np; kp++) {
                if (pthr > 0.f && __ldg(b.prim_bound + kp) * bq < pthr) break;
                float4 Pp, Pa;
                ldg_v8f32(PAf + 8 * (size_t)kp, Pp, Pa);
                const float p = Pp.w, hp = __fdividef(0.5f, p);
                const float pqx = Pp.x - Qp.x, pqy = Pp.y - Qp.y, pqz = Pp.z - Qp.z;
                float u[NR], w[NR];
                if (cache == 2) {
#pragma unroll
                    for (int i = 0; i < NR; i++) {
                        u[i] = cache_u[slot * NR + i];
                        w[i] = cache_w[slot * NR + i];
                    }
                } else {
                    const float rs = rsqrtf(p + q);
                    const float ipq = rs * rs;
                    const float T = p * q * ipq * (pqx * pqx + pqy * pqy + pqz * pqz);
                    rys_eval<NR>(T, thrf, strict, tabf, u, w);
                    const float pref = Pa.w * Qa.w * rs;
#pragma unroll
                    for (int i = 0; i < NR; i++) {
                        u[i] *= ipq;
                        w[i] *= pref;
                        if (cache == 1) {
                            cache_u[slot * NR + i] = u[i];
                            cache_w[slot * NR + i] = w[i];
                        }
                    }
                }
                slot++;
                if constexpr (NR >= 2 && pair_roots_class(LA * 1000 + LB * 100 + LC * 10 + LD)) {
                    // roots in pairs (a last odd root pairs with a zero weight)
                    constexpr int NP = (NR + 1) / 2;
                    float u2[2 * NP], w2[2 * NP];
#pragma unroll
                    for (int i = 0; i < 2 * NP; i++) {
                        u2[i] = i < NR ? u[i] : 0.f;
                        w2[i] = i < NR ? w[i] : 0.f;
                    }
#pragma unroll(FULL ? NP : 1)
                    for (int r = 0; r < NP; r++) {
                        const F2 ui(u2[0], u2[1]), wr(w2[0], w2[1]);
#pragma unroll
                        for (int i = 0; i + 2 < 2 * NP; i++) {  // rotate the next pair to the front
                            u2[i] = u2[i + 2];
                            w2[i] = w2[i + 2];
                        }
                        const F2 fq = F2(q) * ui, fp = F2(p) * ui;
                        const F2 b00 = F2(0.5f) * ui;
                        const F2 b10 = F2(hp) * (F2(1.0f) + F2(-q) * ui), b01 = F2(hq) * (F2(1.0f) + F2(-p) * ui);
                        F2 gx[LAB + 1][LCD + 1], gy[LAB + 1][LCD + 1], gz[LAB + 1][LCD + 1];
                        vrr<LAB, LCD, F2>(gx, F2(Pa.x) + F2(-pqx) * fq, F2(Qa.x) + F2(pqx) * fp, b10, b01, b00, F2(1.0f));
                        vrr<LAB, LCD, F2>(gy, F2(Pa.y) + F2(-pqy) * fq, F2(Qa.y) + F2(pqy) * fp, b10, b01, b00, F2(1.0f));
                        vrr<LAB, LCD, F2>(gz, F2(Pa.z) + F2(-pqz) * fq, F2(Qa.z) + F2(pqz) * fp, b10, b01, b00, wr);
                        if constexpr (HGP) contract_hgp_pair<LA, LB, LC>(gx, gy, gz, acc);
                        else contract_root_pair<LA, LB, LC, LD, NMU>(gx, gy, gz, F2(abx), F2(aby), F2(abz), F2(cdx),
                                                                    F2(cdy), F2(cdz), ex, ey, ez, acc);
                    }
                } else {
#pragma unroll(FULL ? NR : 1)
                for (int r = 0; r < NR; r++) {
                    const float ui = u[0], wr = w[0];
#pragma unroll
                    for (int i = 0; i + 1 < NR; i++) {
                        u[i] = u[i + 1];
                        w[i] = w[i + 1];
                    }
                    const float fq = q * ui, fp = p * ui;
                    const float b00 = 0.5f * ui, b10 = hp * (1.0f - fq), b01 = hq * (1.0f - fp);
                    R gx[LAB + 1][LCD + 1], gy[LAB + 1][LCD + 1], gz[LAB + 1][LCD + 1];
                    vrr<LAB, LCD, R>(gx, Pa.x - fq * pqx, Qa.x + fp * pqx, b10, b01, b00, 1.0f);
                    vrr<LAB, LCD, R>(gy, Pa.y - fq * pqy, Qa.y + fp * pqy, b10, b01, b00, 1.0f);
                    vrr<LAB, LCD, R>(gz, Pa.z - fq * pqz, Qa.z + fp * pqz, b10, b01, b00, wr);
                    if constexpr (HGP) contract_hgp<LA, LB, LC, R>(gx, gy, gz, acc);
                    else contract_root<LA, LB, LC, LD, R, NMU>(gx, gy, gz, abx, aby, abz, cdx, cdy, cdz, ex, ey, ez, acc);
                }
                }
            }
        }
    }
}

// normalisation of a component product: sqrt(3)^n3
__device__ __forceinline__ double s3pow(int n3) {
    return n3 == 0 ? 1.0 : n3 == 1 ? 1.7320508075688772935 : n3 == 2 ? 3.0 : n3 == 3 ? 5.196152422706632 : 9.0;
}
__device__ __forceinline__ int cs3_rt(int l, int c) { return (l == 2 && c >= 3) ? 1 : 0; }

// 0-based packed index of (i, j): max(i,j)(max+1)/2 + min in unsigned 32-bit
// arithmetic, exact for nbf <= 65535: the largest basis whose packed length
// fits the int32 matrix_size of the interface (setup rejects larger ones)
__device__ __forceinline__ unsigned tri0(unsigned i, unsigned j) {
    const unsigned hi = i > j ? i : j, lo = i > j ? j : i;
    return ((hi * (hi + 1u)) >> 1) + lo;
}

// target of a K or J update: the CTA's shared tile (rows of A and B of F) or,
// when the tile does not fit, the packed matrix itself
// (T: the digestion type, double for the FP64 tier and float for the FP32
// tier, whose tile is single precision; F itself is always FP64.)
template <typename T>
struct Rows {
    T *tile;  // rows x nbf, or null
    double *F;
    int nbf;
    __device__ __forceinline__ void add(int r, int bf_row, int col, T v) const {
        if (v == T(0)) return;
        if (tile) atomicAdd(tile + r * nbf + col, v);
        else atomicAdd(F + tri0(bf_row, col), (double)v);
    }
};

template <typename T>
struct QuartetCtx {
    int bfA, bfB, bfC, bfD;
    bool iandj, kandl, same;
    T cut;
    const T *__restrict__ Dm;   // the build's density as a full n x n matrix (the Coulomb terms)
    const T *__restrict__ DmK;  // the density of the exchange terms: Dm itself, or (open-shell builds)
                                // a second n x n matrix
    unsigned ld;                // n
};

// D(i, j) from the full matrix: the row is the CTA's bra shell (A or B) or
// the ket's first shell, the column runs over a shell's components, so one
// shell's components share a sector and every lane of a CTA reads the same
// rows A and B (n <= 65535: i * n + j fits unsigned 32-bit)
template <typename T>
__device__ __forceinline__ T dget(const T *__restrict__ Dm, unsigned ld, unsigned i, unsigned j) {
    return __ldg(Dm + i * ld + j);
}

// Per-class compile-time shape: A components per pass (bounds the contracted
// block held in registers) and resident CTAs per SM requested from the
// register allocator.  The table was tuned offline with ptxas register and
// spill reports; LIBERI_TUNE_* override one class for that search.  The FP64
// resident-CTA counts were measured again, per class, on C60 with the
// shared-memory carveout sized to the resident CTAs and the staged table
// rows (every count from three below to one above the earlier choice):
// (sp|sp) 6 -> 4 (14.10 -> 12.99 ms: no spills, and its table rows out of
// L1), (sp|sd) 5 -> 4 (4.96 -> 4.14), (ss|sd) 6 -> 5 (1.91 -> 1.75), (sd|sd)
// 2 -> 3 (0.73 -> 0.70), (dd|dd) 2 -> 1 (0.45 -> 0.33 ms).
constexpr int class_key(int la, int lb, int lc, int ld) { return la * 1000 + lb * 100 + lc * 10 + ld; }
constexpr int tuned_nmu(int key) {
#ifdef LIBERI_TUNE_KEY
    if (key == LIBERI_TUNE_KEY) return LIBERI_TUNE_NMU;
#endif
    switch (key) {
        case 1000: return 3;
        case 1010: return 3;
        case 1100: return 3;
        case 1110: return 3;
        case 1111: return 1;
        case 1120: return 3;
        case 2000: return 6;
        case 2010: return 6;
        case 2020: return 6;
        case 2100: return 6;
        case 2110: return 6;
        case 2111: return 1;
        case 2120: return 1;
        case 2121: return 1;
        case 2200: return 6;
        case 2210: return 1;
        case 2211: return 1;
        case 2220: return 1;
        case 2221: return 1;
        case 2222: return 1;
        default: return 0;
    }
}
constexpr int tuned_minb(int key) {
#ifdef LIBERI_TUNE_KEY
    if (key == LIBERI_TUNE_KEY) return LIBERI_TUNE_MINB;
#endif
    switch (key) {
        case 0: return 6;
        case 1000: return 6;
        case 1010: return 4;
        case 1100: return 5;
        case 1110: return 4;
        case 1111: return 3;
        case 1120: return 2;
        case 2000: return 5;
        case 2010: return 4;
        case 2020: return 3;
        case 2100: return 4;
        case 2110: return 2;
        case 2111: return 3;
        case 2120: return 3;
        case 2121: return 2;
        case 2200: return 2;
        case 2210: return 3;
        case 2211: return 2;
        case 2220: return 2;
        case 2221: return 2;
        case 2222: return 1;
        default: return 3;
    }
}

// FP32 tier shapes (half the register footprint per value); 0 / default
// falls back to the FP64 choice.  Resident-CTA counts measured again per
// class in the C60 mixed build at cut 1e-2 (every count from three below to
// one above the earlier choice): one more CTA pays in (pp|pp) 3.99 -> 3.80,
// (pd|pp) 6.20 -> 5.91, (ss|sp) 4.19 -> 4.11, (ss|sd) 1.13 -> 1.10 and (pd|sd)
// 2.06 -> 2.02 ms.  LIBERI_TUNE_* with LIBERI_TUNE_F32 override
// one class of this table for the offline search.
constexpr int tuned_nmu_f32(int key) {
#ifdef LIBERI_TUNE_KEY
    if (key == LIBERI_TUNE_KEY) return LIBERI_TUNE_NMU;
#endif
    switch (key) {
        case 0: return 1;
        case 1000: return 3;
        case 1010: return 3;
        case 1100: return 3;
        case 1110: return 3;
        case 1111: return 1;
        case 1120: return 3;
        case 2000: return 6;
        case 2010: return 6;
        case 2020: return 6;
        case 2100: return 6;
        case 2110: return 6;
        case 2111: return 1;
        case 2120: return 2;
        case 2121: return 1;
        case 2200: return 6;
        case 2210: return 2;
        case 2211: return 1;
        case 2220: return 2;
        default: return tuned_nmu(key);
    }
}
constexpr int tuned_minb_f32(int key) {
#ifdef LIBERI_TUNE_KEY
    if (key == LIBERI_TUNE_KEY) return LIBERI_TUNE_MINB;
#endif
    switch (key) {
        case 0: return 8;
        case 1000: return 9;
        case 1010: return 8;
        case 1100: return 8;
        case 1110: return 5;
        case 1111: return 5;
        case 1120: return 3;
        case 2000: return 7;
        case 2010: return 6;
        case 2020: return 4;
        case 2100: return 5;
        case 2110: return 3;
        case 2111: return 5;
        case 2120: return 4;
        case 2121: return 2;
        case 2200: return 3;
        case 2210: return 3;
        case 2211: return 2;
        case 2220: return 2;
        case 2222: return 2;
        default: return tuned_minb(key);
    }
}

// Alternative shapes per class and precision (variants 1..NVARIANT-1), chosen
// at run time by the autotuner; 0 in a table means "same as variant 0".
// Alternative shapes (variants 1, 2) per class and precision from the
// ptxas register/spill search: higher resident-CTA counts at the price of
// some spills (measured: occupancy pays more than spills cost, extra passes
// never pay); variant 0 is the default above, chosen by measurement.
// Key: class key * 10 + variant; 0 = same as variant 0.
constexpr int alt_nmu(int key, bool f32, int v) {
    if (f32) {
        switch (key * 10 + v) {
            case 11001: return 3;
            case 11101: return 3;
            case 11102: return 3;
            case 11111: return 3;
            case 11112: return 3;
            case 21101: return 6;
            case 21111: return 3;
            case 21112: return 3;
            case 21211: return 1;
            default: return 0;
        }
    }
    switch (key * 10 + v) {
        case 10001: return 3;
        case 10101: return 3;
        case 10102: return 3;
        case 11001: return 3;
        case 11002: return 3;
        case 11101: return 3;
        case 21101: return 6;
        default: return 0;
    }
}
constexpr int alt_minb(int key, bool f32, int v) {
    if (f32) {
        switch (key * 10 + v) {
            case 11001: return 6;
            case 11101: return 6;
            case 11102: return 8;
            case 11111: return 3;
            case 11112: return 3;
            case 21101: return 4;
            case 21111: return 2;
            case 21112: return 3;
            case 21211: return 3;
            default: return 0;
        }
    }
    switch (key * 10 + v) {
        case 10001: return 8;
        case 10101: return 5;
        case 10102: return 6;
        case 11001: return 5;
        case 11002: return 6;
        case 11101: return 3;
        case 21101: return 3;
        default: return 0;
    }
}

// Threads per quartet of a shape variant (multi-pass classes): G lanes of a
// warp share one quartet and take its passes over the A components in turn
// (lane g: passes g, g+G, ...), so a quartet's passes run side by side
// instead of one after another; 1 = one thread per quartet.  Variants 1 and
// 2 of the multi-pass classes that have no other alternative shape.
// Variant 0 (the default): (dd|dd) in FP64 runs two lanes per quartet (its
// 1,830 C60 quartets: 0.73 -> 0.45 ms); variant 1 keeps one.
constexpr int tuned_tpq(int key, bool f32) { return (!f32 && key == 2222) ? 2 : 1; }
constexpr int alt_tpq(int key, bool f32, int v) {
    if (v == 0) return tuned_tpq(key, f32);
    if (!f32 && key == 2222) return v == 1 ? 1 : 4;
    if (f32) {
        switch (key * 10 + v) {
            case 21201: case 21212: case 22101: case 22111: case 22201: case 22211: case 22221: return 2;
            case 21202: case 22102: case 22112: case 22202: case 22212: case 22222: return 4;
            default: return 1;
        }
    }
    switch (key) {
        case 1111: case 2111: case 2120: case 2121: case 2210: case 2211: case 2220: case 2221: case 2222:
            return v == 1 ? 2 : 4;
        default: return 1;
    }
}

template <int LA, int LB, int LC, int LD, typename R, int V = 0>
struct PassShape {
    static constexpr bool F32 = std::is_same<R, float>::value;
    static constexpr int KEY = class_key(LA, LB, LC, LD);
    static constexpr int PER_MU = ncart(LB) * ncart(LC) * ncart(LD);
    static constexpr int NA = ncart(LA);
    static constexpr int NMU_DEF = PER_MU >= 40 ? 1 : (40 / PER_MU);
    static constexpr int NMU_V0 = F32 ? tuned_nmu_f32(KEY) : tuned_nmu(KEY);
    static constexpr int NMU_TUNED = (V > 0 && alt_nmu(KEY, F32, V) > 0) ? alt_nmu(KEY, F32, V) : NMU_V0;
    static constexpr int NMU_T = NMU_TUNED > 0 ? NMU_TUNED : NMU_DEF;
    static constexpr int NMU = NMU_T > NA ? NA : NMU_T;
    static constexpr int NPASS = (NA + NMU - 1) / NMU;
    static constexpr int MINB_V0 = F32 ? tuned_minb_f32(KEY) : tuned_minb(KEY);
    static constexpr int MINB = (V > 0 && alt_minb(KEY, F32, V) > 0) ? alt_minb(KEY, F32, V) : MINB_V0;
    // threads per quartet (powers of two; only where the class has passes to share)
    static constexpr int TPQ = NPASS > 1 ? alt_tpq(KEY, F32, V) : 1;
    // a variant is compiled only when it differs from variant 0
    static constexpr bool DISTINCT = V == 0 || NMU != PassShape<LA, LB, LC, LD, R, 0>::NMU ||
                                     MINB != PassShape<LA, LB, LC, LD, R, 0>::MINB ||
                                     TPQ != PassShape<LA, LB, LC, LD, R, 0>::TPQ;
};

constexpr int CLASS_THREADS = 128;
// dynamic shared memory a class CTA may request (below the 227 KB per-CTA
// limit, leaving room for static shared memory)
constexpr int CLASS_DYN_SMEM_MAX = 226 * 1024;
constexpr int ROOT_CACHE_PQ = 32;  // primitive quartets per shell quartet whose roots are kept across passes
// classes whose passes reuse the roots (measured per class on C60: the FP64
// multi-pass classes except (pd|pd); FP32 gains nothing)
constexpr bool root_cache_on(int key, bool f32) { return !f32 && key != 2121; }

// Per-quartet partial sums that outlive a pass: K updates of the B rows
// (bc[ib][ic], bd[ib][id]) and the ket-pair J block (cd[ic][id]).  Single-
// pass classes keep them in registers; multi-pass classes in per-thread
// shared-memory slots (stride CLASS_THREADS, bank-conflict free).
template <int NB, int NC, int ND, bool SM, typename T>
struct KBuf {
    static constexpr int N = NB * NC + NB * ND + NC * ND;
    T r[SM ? 1 : N];
    T *s;
    __device__ __forceinline__ T &at(int i) {
        if constexpr (SM) return s[i * CLASS_THREADS];
        else return r[i];
    }
    __device__ __forceinline__ T &bc(int ib, int ic) { return at(ib * NC + ic); }
    __device__ __forceinline__ T &bd(int ib, int id) { return at(NB * NC + ib * ND + id); }
    __device__ __forceinline__ T &cd(int ic, int id) { return at(NB * NC + NB * ND + ic * ND + id); }
};

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// sum over the lanes that share lane % G (G a power of two)
template <int G, typename T>
__device__ __forceinline__ T warp_sum_strided(T v) {
#pragma unroll
    for (int o = 16; o >= G; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// sum over the G lanes of one group (lanes that differ in the low bits only)
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Digestion of one A component (row mu) of a quartet whose four shells give
// distinct function pairs (no identical shells in the bra or the ket, bra !=
// ket): every Cartesian component is unique and no 0.5 factor applies
// (int0000.F90:255-292 reduce to the plain six updates), so the D sub-blocks
// are loaded once per pass and each integral costs one cut select and six
// FMAs.  jab returns 4 sum D(la,si) (mu nu|la si) for the warp-level J
// reduction of the row pair.
template <int LA, int LB, int LC, int LD, typename R, typename KB>
__device__ __forceinline__ void digest_row_distinct(const R (&a)[ncart(LB)][ncart(LC)][ncart(LD)], int ia,
                                                    const QuartetCtx<R> &qc,
                                                    const R (&dCD)[ncart(LC)][ncart(LD)],
                                                    const R (&dBD)[ncart(LB)][ncart(LD)],
                                                    const R (&dBC)[ncart(LB)][ncart(LC)], const Rows<R> &rows,
                                                    KB &kb, R (&jab)[ncart(LB)]) {
    constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    const R *__restrict__ Dm = qc.Dm;
    const int mu = qc.bfA + ia;
    const R sa = R(s3pow(cs3_rt(LA, ia)));
    R dAB[NB], dAC[NC], dAD[ND];
#pragma unroll
    for (int ib = 0; ib < NB; ib++) dAB[ib] = R(4) * dget(Dm, qc.ld, mu, qc.bfB + ib);
#pragma unroll
    for (int ic = 0; ic < NC; ic++) dAC[ic] = dget(qc.DmK, qc.ld, mu, qc.bfC + ic);
#pragma unroll
    for (int id = 0; id < ND; id++) dAD[id] = dget(qc.DmK, qc.ld, mu, qc.bfD + id);
    R kac[NC], kad[ND];
#pragma unroll
    for (int ib = 0; ib < NB; ib++) jab[ib] = R(0);
#pragma unroll
    for (int ic = 0; ic < NC; ic++) kac[ic] = R(0);
#pragma unroll
    for (int id = 0; id < ND; id++) kad[id] = R(0);
#pragma unroll
    for (int ib = 0; ib < NB; ib++)
#pragma unroll
        for (int ic = 0; ic < NC; ic++)
#pragma unroll
            for (int id = 0; id < ND; id++) {
                R v = a[ib][ic][id] * (sa * R(s3pow(cs3(LB, ib) + cs3(LC, ic) + cs3(LD, id))));
                v = fabs(v) < qc.cut ? R(0) : v;
                jab[ib] = fma(v, dCD[ic][id], jab[ib]);
                kb.cd(ic, id) = fma(v, dAB[ib], kb.cd(ic, id));
                kac[ic] = fma(v, dBD[ib][id], kac[ic]);
                kad[id] = fma(v, dBC[ib][ic], kad[id]);
                kb.bc(ib, ic) = fma(v, dAD[id], kb.bc(ib, ic));
                kb.bd(ib, id) = fma(v, dAC[ic], kb.bd(ib, id));
            }
#pragma unroll
    for (int ib = 0; ib < NB; ib++) jab[ib] *= R(4);
#pragma unroll
    for (int ic = 0; ic < NC; ic++) rows.add(ia, mu, qc.bfC + ic, -kac[ic]);
#pragma unroll
    for (int id = 0; id < ND; id++) rows.add(ia, mu, qc.bfD + id, -kad[id]);
}

// Digestion of one A component with the reference's unique-component loops
// and 0.5 factors (identical shells in the bra or the ket, or bra == ket).
template <int LA, int LB, int LC, int LD, typename R, typename KB>
__device__ __forceinline__ void digest_row_general(const R (&a)[ncart(LB)][ncart(LC)][ncart(LD)], int ia,
                                                   const QuartetCtx<R> &qc, const Rows<R> &rows, KB &kb,
                                                   R (&jab)[ncart(LB)]) {
    constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr bool can_same = (LA == LC) && (LB == LD);
    const int mu = qc.bfA + ia;
    const int n3a = cs3_rt(LA, ia);
    R kac[NC], kad[ND];
#pragma unroll
    for (int ic = 0; ic < NC; ic++) kac[ic] = R(0);
#pragma unroll
    for (int id = 0; id < ND; id++) kad[id] = R(0);
#pragma unroll
    for (int ib = 0; ib < NB; ib++) {
        jab[ib] = R(0);
        if (LA == LB && qc.iandj && ib > ia) continue;
        const int nu = qc.bfB + ib;
        const R dmn = dget(qc.Dm, qc.ld, mu, nu);
#pragma unroll
        for (int ic = 0; ic < NC; ic++) {
            const int la = qc.bfC + ic;
#pragma unroll
            for (int id = 0; id < ND; id++) {
                if (LC == LD && qc.kandl && id > ic) continue;
                if (can_same && qc.same) {
                    const int oij = qc.iandj ? ia * (ia + 1) / 2 + ib : ia * NB + ib;
                    const int okl = qc.kandl ? ic * (ic + 1) / 2 + id : ic * ND + id;
                    if (okl > oij) continue;
                }
                R v = a[ib][ic][id] * R(s3pow(n3a + cs3(LB, ib) + cs3(LC, ic) + cs3(LD, id)));
                if (fabs(v) < qc.cut) continue;
                const int si = qc.bfD + id;
                // 0.5 factors for coinciding function indices (int0000.F90:288-292)
                if (mu == nu) v *= R(0.5);
                if (la == si) v *= R(0.5);
                if ((mu == la && nu == si) || (mu == si && nu == la)) v *= R(0.5);
                jab[ib] += R(4) * v * dget(qc.Dm, qc.ld, la, si);
                kb.cd(ic, id) += R(4) * v * dmn;
                kac[ic] += v * dget(qc.DmK, qc.ld, nu, si);
                kad[id] += v * dget(qc.DmK, qc.ld, nu, la);
                kb.bc(ib, ic) += v * dget(qc.DmK, qc.ld, mu, si);
                kb.bd(ib, id) += v * dget(qc.DmK, qc.ld, mu, la);
            }
        }
    }
#pragma unroll
    for (int ic = 0; ic < NC; ic++) rows.add(ia, mu, qc.bfC + ic, -kac[ic]);
#pragma unroll
    for (int id = 0; id < ND; id++) rows.add(ia, mu, qc.bfD + id, -kad[id]);
}

// Digestion of one pass of M A components (from mu0): the D sub-blocks of a
// distinct-shell quartet, the digestion of each component, and the row
// pair's J summed over the lanes that hold the same component (all lanes of
// the warp for G = 1, every G-th lane otherwise) and added once.  Every lane
// reaches the reductions (the quartet loop is warp-uniform; idle lanes, and
// for G > 1 trips past a lane's passes (live false), digest zeros).
template <int LA, int LB, int LC, int LD, typename R, int M, bool HGP, int G, typename ACC, typename KB>
__device__ __forceinline__ void digest_pass(const ACC &acc, int mu0, bool live, R abx, R aby, R abz,
                                            const QuartetCtx<R> &qc, const Rows<R> &rows, KB &kb) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    const bool distinct = !qc.iandj && !qc.kandl && !qc.same;
    R dCD[NC][ND], dBD[NB][ND], dBC[NB][NC];
    if (distinct) {
#pragma unroll
        for (int ic = 0; ic < NC; ic++)
#pragma unroll
            for (int id = 0; id < ND; id++) dCD[ic][id] = dget(qc.Dm, qc.ld, qc.bfC + ic, qc.bfD + id);
#pragma unroll
        for (int ib = 0; ib < NB; ib++) {
#pragma unroll
            for (int id = 0; id < ND; id++) dBD[ib][id] = dget(qc.DmK, qc.ld, qc.bfB + ib, qc.bfD + id);
#pragma unroll
            for (int ic = 0; ic < NC; ic++) dBC[ib][ic] = dget(qc.DmK, qc.ld, qc.bfB + ib, qc.bfC + ic);
        }
    }
#pragma unroll
    for (int m = 0; m < M; m++) {
        const int ia = mu0 + m;
        if constexpr (G == 1) {
            if (ia >= NA) break;
        }
        const bool comp = G == 1 || (live && ia < NA);
        R jab[NB];
        if constexpr (G > 1) {
#pragma unroll
            for (int ib = 0; ib < NB; ib++) jab[ib] = R(0);
        }
        if (comp) {
            if constexpr (HGP) {
                // one pass: the component index is the unrolled m (a compile-time
                // index into acc; the run-time ia would put acc in local memory)
                R sl[NB][NC][ND];
                bra_transfer<LA, LB, LC, R>(acc, m, abx, aby, abz, sl);
                if (distinct)
                    digest_row_distinct<LA, LB, LC, LD, R>(sl, ia, qc, dCD, dBD, dBC, rows, kb, jab);
                else
                    digest_row_general<LA, LB, LC, LD, R>(sl, ia, qc, rows, kb, jab);
            } else {
                if (distinct)
                    digest_row_distinct<LA, LB, LC, LD, R>(acc[m], ia, qc, dCD, dBD, dBC, rows, kb, jab);
                else
                    digest_row_general<LA, LB, LC, LD, R>(acc[m], ia, qc, rows, kb, jab);
            }
        }
#pragma unroll
        for (int ib = 0; ib < NB; ib++) jab[ib] = warp_sum_strided<G>(jab[ib]);
        if ((int)(threadIdx.x & 31) < G && comp) {
#pragma unroll
            for (int ib = 0; ib < NB; ib++) rows.add(ia, qc.bfA + ia, qc.bfB + ib, jab[ib]);
        }
    }
}

// Runtime loop over passes of NMU A components; digestion of each pass.
template <int LA, int LB, int LC, int LD, typename R, int V, typename KB>
__device__ __forceinline__ void run_passes(const DevBasis &b, int p0, int np, int q0, int nq, const double4 &A,
                                           const double4 &C, R abx, R aby, R abz, R cdx, R cdy, R cdz,
                                           double thr, bool strict, const double *__restrict__ tab,
                                           const float *__restrict__ tabf, const QuartetCtx<R> &qc,
                                           const Rows<R> &rows, KB &kb, float pthr, float bpmax,
                                           const double *stab) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    using PS = PassShape<LA, LB, LC, LD, R, V>;
    constexpr int M = PS::NMU;
    // Multi-pass classes evaluate the Rys roots and weights of each primitive
    // quartet once: pass 0 keeps them (scaled) in a per-thread local array,
    // later passes read them back (coalesced across the warp) instead of
    // gathering table coefficients again; quartets with more primitive
    // quartets than the array holds recompute them.
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    constexpr bool CACHE = PS::NPASS > 1 && root_cache_on(PS::KEY, PS::F32);
    constexpr int CAP = CACHE ? ROOT_CACHE_PQ : 1;
    R cache_u[CAP * NR], cache_w[CAP * NR];
    const bool cache_ok = CACHE && np * nq <= CAP;
    constexpr bool HGP = hgp_class<LA, LB, LC, LD>(PS::NPASS);
    using Acc = typename std::conditional<HGP, R[nrange(LA, LA + LB)][NC], R[M][NB][NC][ND]>::type;
    // G lanes per quartet (lane g of a group takes passes g, g+G, ...)
    constexpr int G = PS::TPQ;
    if constexpr (G == 1) {
#pragma unroll 1
        for (int pass = 0; pass < PS::NPASS; pass++) {
            const int mu0 = pass * M;
            // (e0|c0) intermediates (HGP) or the (ab|cd) block of this pass's A components
            Acc acc;
            eval_block<LA, LB, LC, LD, R, M, HGP>(b, p0, np, q0, nq, A, C, abx, aby, abz, cdx, cdy, cdz, thr, strict,
                                                  tab, tabf, mu0, acc, cache_u, cache_w,
                                                  cache_ok ? (pass == 0 ? 1 : 2) : 0, pthr, bpmax, stab);
            digest_pass<LA, LB, LC, LD, R, M, HGP, 1>(acc, mu0, true, abx, aby, abz, qc, rows, kb);
        }
    } else {
        // every lane runs the same number of trips; a trip past a lane's last
        // pass evaluates and digests nothing, but still joins the warp sums
        constexpr int NIT = (PS::NPASS + G - 1) / G;
        const int sub = (int)(threadIdx.x & 31) & (G - 1);
#pragma unroll 1
        for (int trip = 0; trip < NIT; trip++) {
            const int pass = trip * G + sub;
            const bool live = pass < PS::NPASS;
            const int mu0 = (live ? pass : 0) * M;
            Acc acc;
            eval_block<LA, LB, LC, LD, R, M, HGP>(b, p0, np, q0, live ? nq : 0, A, C, abx, aby, abz, cdx, cdy, cdz,
                                                  thr, strict, tab, tabf, mu0, acc, cache_u, cache_w,
                                                  cache_ok ? (trip == 0 ? 1 : 2) : 0, pthr, bpmax, stab);
            digest_pass<LA, LB, LC, LD, R, M, HGP, G>(acc, mu0, live, abx, aby, abz, qc, rows, kb);
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
    const float *tabf;
    const double *Dm;        // this build's D as a full n x n matrix
    const float *Dmf;        // FP32 tier: the same in single precision
    double *F;
    double cut;
    double thr;
    bool strict;
    const int4 *tasks;       // (bra position, first ket position, ket count, -)
    const int *ntasks_dev;   // device task count (per-build task lists) or null
    int ntasks;              // static task count / grid bound
    int nbf;
    int tile_rows;           // 1: stage rows of A and B of F in shared memory
    const int *bra_ids, *ket_ids, *bra_orig, *ket_orig;
    const double4 *ket_rec;  // ket records (KET_REC per ket position)
    int swapped;             // plan bra list is the reference's ket list
    RankSplit rs;
    const MolView *mols;     // batched launch: per-molecule data (task.w), else null
    const ClassView *cviews; // batched launch: per-molecule lists of this class
    const unsigned long long *maxd;  // FP32 tier: max|D| bits (per molecule for batches)
    size_t k_offset;                 // exchange density at D + k_offset (0: D itself; n*n for open-shell builds)
    double prim_cut;                 // FP32 tier: primitive screening cut (0 = off)
};

// Does this rank evaluate the quartet (bra position ibra, ket position j) under
// the reference's rank split?  The flat iteration index of the reference
// kernel from the positions in its compacted lists (int0001.F90:117,
// int2211_rysgen.F90:351, triangle kernels by bra position).
__device__ __forceinline__ bool quartet_owned(const ClassArgs &a, int ibra, int j) {
    if (a.rs.nsize <= 1) return true;
    long long bo = a.bra_orig[ibra], ko = a.ket_orig[j];
    if (a.swapped) { long long tmp = bo; bo = ko; ko = tmp; }
    long long it;
    if (a.rs.tri) it = (bo > ko ? bo : ko) + 1;
    else if (a.rs.ketmajor) it = ko * a.rs.nbra_ref + bo + 1;
    else it = bo * a.rs.nket_ref + ko + 1;
    return rank_owns(a.rs, it);
}

// Per-molecule data of a task.  A single-molecule launch reads the kernel
// parameters at every use (constant-bank operands, no registers held across
// the quartet loop); a batched launch reads the task's molecule view (task.w).
template <bool BATCH>
__device__ __forceinline__ const DevBasis &mol_basis(const ClassArgs &a, int w) {
    if constexpr (BATCH) return a.mols[w].b; else return a.b;
}
template <bool BATCH, typename T>
__device__ __forceinline__ const T *mol_D(const ClassArgs &a, int w) {
    if constexpr (std::is_same<T, float>::value) return BATCH ? a.mols[w].Df : a.Dmf;  // FP32 tier
    else if constexpr (BATCH) return a.mols[w].Dsq;
    else return a.Dm;
}
template <bool BATCH>
__device__ __forceinline__ double *mol_F(const ClassArgs &a, int w) {
    if constexpr (BATCH) return a.mols[w].F; else return a.F;
}
template <bool BATCH>
__device__ __forceinline__ int mol_nbf(const ClassArgs &a, int w) {
    if constexpr (BATCH) return a.mols[w].nbf; else return a.nbf;
}
template <bool BATCH>
__device__ __forceinline__ const int *mol_bra(const ClassArgs &a, int w) {
    if constexpr (BATCH) return a.cviews[w].bra_ids; else return a.bra_ids;
}
template <bool BATCH>
__device__ __forceinline__ const double4 *mol_ketrec(const ClassArgs &a, int w) {
    if constexpr (BATCH) return a.cviews[w].ket_rec; else return a.ket_rec;
}

// One CTA task: row pair t.x against kets t.y .. t.y+t.z-1 of one molecule.
template <int LA, int LB, int LC, int LD, typename R, bool BATCH, int V>
__device__ __forceinline__ void class_task(const ClassArgs &a, const int4 t) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    extern __shared__ __align__(16) unsigned char class_smem[];
    // the class's staged table rows come first (16-byte aligned), then the
    // F-row tile and the per-thread slots (batched launches do not stage)
    constexpr size_t STB = BATCH ? 0 : stab_bytes<LA, LB, LC, LD, R>();
    const double *stab = nullptr;
    if constexpr (STB > 0) {
        constexpr int NRt = (LA + LB + LC + LD) / 2 + 1;
        double *st = reinterpret_cast<double *>(class_smem);
        const double *g = a.tab + rys_table_off(NRt);
        for (int i = threadIdx.x; i < STAB_NINT * 16 * NRt; i += CLASS_THREADS) {
            const int kk = i / (16 * NRt), j = i - kk * 16 * NRt;
            st[kk * stab_stride(NRt) + j] = __ldg(g + i);
        }
        __syncthreads();
        // rows 0..100 cover T <= 25: the class's large-T form takes every T above
        if (a.thr <= 25.0) stab = st;
    }
    R *tile = reinterpret_cast<R *>(class_smem + STB);  // the digestion type: FP32 tile for the FP32 tier
    const int ibra = t.x, k0 = t.y, cnt = t.z;
    const DevBasis &bas = mol_basis<BATCH>(a, t.w);
#define LIBERI_D mol_D<BATCH, R>(a, t.w)
#define LIBERI_F mol_F<BATCH>(a, t.w)
#define LIBERI_NBF mol_nbf<BATCH>(a, t.w)
    const int P = __ldg(mol_bra<BATCH>(a, t.w) + ibra);
    const int2 sab = bas.pair_shell[P];
    const double4 A = bas.shell_xyz[sab.x], B = bas.shell_xyz[sab.y];
    const int bfA = bas.shell_bf0[sab.x], bfB = bas.shell_bf0[sab.y];
    const int nrow = NA + NB;
    // the F-row tile pays for its zeroing and flush (2 (NA+NB) nbf shared
    // accesses) only when the task's kets touch a fair part of each row;
    // short tasks (the FP64 head of a mixed-precision item, item tails) add
    // their K updates to F directly
    const bool use_tile = a.tile_rows != 0 && 4 * cnt * (NC + ND) >= LIBERI_NBF;
    if (use_tile) {
        for (int i = threadIdx.x; i < nrow * LIBERI_NBF; i += CLASS_THREADS) tile[i] = R(0);
        __syncthreads();
    }
    R *slots = tile + (use_tile ? nrow * LIBERI_NBF : 0);  // per-thread partial sums (multi-pass)
    Rows<R> rowsA{use_tile ? tile : nullptr, LIBERI_F, LIBERI_NBF};
    Rows<R> rowsB{use_tile ? tile + NA * LIBERI_NBF : nullptr, LIBERI_F, LIBERI_NBF};
    const R abx = R(A.x - B.x), aby = R(A.y - B.y), abz = R(A.z - B.z);
    const int p0 = bas.pair_prim0[P], np = bas.pair_nprim[P];
    // FP32 tier: the task's primitive screening threshold and the largest
    // primitive bound of its bra pair (its first primitive)
    float pthr = 0.f, bpmax = 0.f;
    if constexpr (std::is_same<R, float>::value) {
        if (a.prim_cut > 0.0 && a.maxd && bas.prim_bound) {
            const double md = __longlong_as_double((long long)a.maxd[BATCH ? t.w : 0]);
            if (md > 0.0 && np > 0) {
                pthr = (float)(a.prim_cut / md);
                bpmax = __ldg(bas.prim_bound + p0);  // primitives in order of decreasing bound
            }
        }
    }
    // Warp-uniform loop: every lane of a warp runs the same iterations (the
    // digestion sums the row pair's J over the warp); a lane past the end of
    // the task, or holding a quartet of another rank, evaluates no primitives
    // and digests zeros.  With G threads per quartet a warp takes 32/G
    // quartets per trip, lanes 0..G-1 the first, and so on.
    constexpr int G = PassShape<LA, LB, LC, LD, R, V>::TPQ;
    const int gsub = (int)(threadIdx.x & 31) & (G - 1);
    for (int qb = (int)(threadIdx.x >> 5) * (32 / G); qb < cnt; qb += CLASS_THREADS / G) {
        const int qi = qb + (int)(threadIdx.x & 31) / G;
        bool act = qi < cnt;
        const int j = k0 + (act ? qi : 0);
        if (act && a.rs.nsize > 1) act = quartet_owned(a, ibra, j);
        const double4 *krec = mol_ketrec<BATCH>(a, t.w) + KET_REC * j;
        const double4 r0 = ldg_double4(krec), r1 = ldg_double4(krec + 1);
        const double4 C = make_double4(r0.w, r1.x, r1.y, 0.0);
        const R cdx = R(r0.x), cdy = R(r0.y), cdz = R(r0.z);
        const unsigned long long kbf = (unsigned long long)__double_as_longlong(r1.z);
        const unsigned long long kpr = (unsigned long long)__double_as_longlong(r1.w);
        QuartetCtx<R> qc;
        qc.bfA = bfA; qc.bfB = bfB;
        qc.bfC = (int)(unsigned)kbf; qc.bfD = (int)(unsigned)(kbf >> 32);
        // shells have distinct first functions: same shells <=> same first functions
        qc.iandj = sab.x == sab.y; qc.kandl = qc.bfC == qc.bfD; qc.same = bfA == qc.bfC && bfB == qc.bfD;
        qc.cut = R(a.cut); qc.Dm = LIBERI_D; qc.ld = (unsigned)LIBERI_NBF;
        qc.DmK = LIBERI_D + a.k_offset;  // open-shell builds: the exchange density follows D
        constexpr bool SM = PassShape<LA, LB, LC, LD, R, V>::NPASS > 1;
        KBuf<NB, NC, ND, SM, R> kb;
        kb.s = slots + threadIdx.x;
#pragma unroll
        for (int i = 0; i < KBuf<NB, NC, ND, SM, R>::N; i++) kb.at(i) = R(0);
        run_passes<LA, LB, LC, LD, R, V>(bas, p0, np, (int)(unsigned)kpr, act ? (int)(unsigned)(kpr >> 32) : 0, A, C, abx, aby,
                                      abz, cdx, cdy, cdz, a.thr, a.strict, a.tab, a.tabf, qc, rowsA, kb, pthr, bpmax, stab);
        if constexpr (G > 1) {
            // the group's lanes hold partial sums over their passes: combine
            // them, the group's first lane adds them to F
#pragma unroll
            for (int i = 0; i < KBuf<NB, NC, ND, SM, R>::N; i++) kb.at(i) = group_sum<G>(kb.at(i));
        }
        if (G == 1 || gsub == 0) {
#pragma unroll
            for (int ib = 0; ib < NB; ib++) {
#pragma unroll
                for (int ic = 0; ic < NC; ic++) rowsB.add(ib, bfB + ib, qc.bfC + ic, -kb.bc(ib, ic));
#pragma unroll
                for (int id = 0; id < ND; id++) rowsB.add(ib, bfB + ib, qc.bfD + id, -kb.bd(ib, id));
            }
#pragma unroll
            for (int ic = 0; ic < NC; ic++)
#pragma unroll
                for (int id = 0; id < ND; id++) {
                    const R v = kb.cd(ic, id);
                    if (v != R(0)) atomicAdd(LIBERI_F + tri0(qc.bfC + ic, qc.bfD + id), (double)v);
                }
        }
    }
    if (use_tile) {
        __syncthreads();
        for (int i = threadIdx.x; i < nrow * LIBERI_NBF; i += CLASS_THREADS) {
            const R v = tile[i];
            if (v == R(0)) continue;
            const int r = i / LIBERI_NBF, col = i - r * LIBERI_NBF;
            const int bf = r < NA ? bfA + r : bfB + (r - NA);
            atomicAdd(LIBERI_F + tri0(bf, col), (double)v);
        }
    }
#undef LIBERI_D
#undef LIBERI_F
#undef LIBERI_NBF
}

// BATCH: the task's w field selects the molecule (basis, D, F, plan lists);
// the launch sized the shared-memory tile for the largest molecule.
template <int LA, int LB, int LC, int LD, typename R, bool BATCH, int V>
__global__ void __launch_bounds__(CLASS_THREADS, PassShape<LA, LB, LC, LD, R, V>::MINB) class_kernel(ClassArgs a) {
    const int ntasks = a.ntasks_dev ? *a.ntasks_dev : a.ntasks;
    if ((int)blockIdx.x >= ntasks) return;  // lists counted on the device launch their capacity
    class_task<LA, LB, LC, LD, R, BATCH, V>(a, a.tasks[blockIdx.x]);
}

// sqrt(max |(ab|ab)|) over the components of one pair, for the Schwarz table.
// (primitive pairs p0 .. p0+np-1 of pair P: all of them for the pair's
// Schwarz value, one for the bound of a single primitive pair)
template <int LA, int LB>
__device__ __forceinline__ double schwarz_diag(const DevBasis &b, int P, const double *tab, int p0, int np) {
    constexpr int NA = ncart(LA), NB = ncart(LB);
    const int2 sab = b.pair_shell[P];
    const double4 A = b.shell_xyz[sab.x], B = b.shell_xyz[sab.y];
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    double m = 0.0;
#pragma unroll 1
    for (int ia = 0; ia < NA; ia++) {
        double acc[1][NB][NA][NB];
        eval_block<LA, LB, LA, LB, double, 1, false>(b, p0, np, p0, np, A, A, abx, aby, abz, abx, aby, abz, RYS_TMAX,
                                              false, tab, nullptr, ia, acc, nullptr, nullptr, 0);
#pragma unroll
        for (int ib = 0; ib < NB; ib++) {
            double v = 0.0;
#pragma unroll
            for (int ic = 0; ic < NA; ic++) v = (ic == ia) ? acc[0][ib][ic][ib] : v;
            v = fabs(v) * s3pow(2 * (cs3_rt(LA, ia) + cs3(LB, ib)));
            m = v > m ? v : m;
        }
    }
    return sqrt(m);
}

template <int LA, int LB, int LC, int LD, typename R, bool BATCH, int V>
cudaError_t launch_shape(const ClassArgs &a, cudaStream_t st) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr bool SM = PassShape<LA, LB, LC, LD, R, V>::NPASS > 1;
    const size_t slot_bytes = SM ? (size_t)KBuf<NB, NC, ND, true, R>::N * CLASS_THREADS * sizeof(R) : 0;
    // the F-row tile is staged only when it fits beside the slots (227 KB per CTA)
    const size_t tile_bytes = (size_t)(NA + NB) * a.nbf * sizeof(R);
    // The F-row tile is staged only when it fits beside the slots at the
    // resident-CTA count the register budget allows: a tile that cut
    // occupancy below it (and shrank L1, where spills live) costs more than
    // the global atomics it saves.
    constexpr int MINB = PassShape<LA, LB, LC, LD, R, V>::MINB;
    ClassArgs args = a;
    constexpr size_t STB = BATCH ? 0 : stab_bytes<LA, LB, LC, LD, R>();
    args.tile_rows = (a.tile_rows && (tile_bytes + slot_bytes + STB) * MINB <= CLASS_DYN_SMEM_MAX) ? 1 : 0;
    const size_t smem = (args.tile_rows ? tile_bytes : 0) + slot_bytes + STB;
    // the opt-in limit is raised to the per-CTA maximum, not to this launch's
    // size: a captured graph may hold a larger launch
    cudaError_t e = cudaFuncSetAttribute(class_kernel<LA, LB, LC, LD, R, BATCH, V>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, CLASS_DYN_SMEM_MAX);
    if (e != cudaSuccess) return e;
    // the rest of the SM's 256 KB stays L1 (the class's Rys table rows, pair
    // data and D): a shared-memory carveout of what MINB resident CTAs use
    {
        const size_t need = smem * (size_t)MINB;
        const int carve = need == 0 ? 0 : (int)std::min<size_t>(100, (need * 100 + 228 * 1024 - 1) / (228 * 1024));
        e = cudaFuncSetAttribute(class_kernel<LA, LB, LC, LD, R, BATCH, V>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (e != cudaSuccess) return e;
    }
    class_kernel<LA, LB, LC, LD, R, BATCH, V><<<(unsigned)a.ntasks, CLASS_THREADS, smem, st>>>(args);
    return cudaGetLastError();
}

template <int LA, int LB, int LC, int LD, typename R>
cudaError_t launch_variant(const ClassArgs &a, int variant, cudaStream_t st) {
    if (variant == 1 && PassShape<LA, LB, LC, LD, R, 1>::DISTINCT) {
        if constexpr (PassShape<LA, LB, LC, LD, R, 1>::DISTINCT) return launch_shape<LA, LB, LC, LD, R, false, 1>(a, st);
    }
    if (variant == 2 && PassShape<LA, LB, LC, LD, R, 2>::DISTINCT) {
        if constexpr (PassShape<LA, LB, LC, LD, R, 2>::DISTINCT) return launch_shape<LA, LB, LC, LD, R, false, 2>(a, st);
    }
    return launch_shape<LA, LB, LC, LD, R, false, 0>(a, st);
}

// precision 0: FP64, 1: FP32; variant: shape variant (0..NVARIANT-1; a
// variant identical to 0 runs 0); batched launches run variant 0.
template <int LA, int LB, int LC, int LD>
cudaError_t launch_t(const ClassArgs &a, int precision, int variant, cudaStream_t st) {
    if (a.ntasks <= 0) return cudaSuccess;
    if (a.mols) {
        if (precision == 0) return launch_shape<LA, LB, LC, LD, double, true, 0>(a, st);
        return launch_shape<LA, LB, LC, LD, float, true, 0>(a, st);
    }
    if (precision == 0) return launch_variant<LA, LB, LC, LD, double>(a, variant, st);
    return launch_variant<LA, LB, LC, LD, float>(a, variant, st);
}

}  // namespace liberi
