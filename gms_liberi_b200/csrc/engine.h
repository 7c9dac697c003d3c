// engine.h -- internal structures of the B200 Fock-build engine.
//
// Host side (host.cpp) builds, once per geometry, the device-resident shell,
// pair and quartet-plan buffers described here; the device side (kernels.cu)
// evaluates the 21 s/p/d quartet classes of the reference driver
// (src/liberi_driver.F90:69-102) with Rys quadrature and digests them into
// the packed Fock matrix.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace liberi {

constexpr int NKERN = 21;
constexpr int MAXROOT = 5;
// Rys tables: intervals of width 1 in T on [0, RYS_TMAX), 13 power-basis
// coefficients per function in x = 2(T - k) - 1.
constexpr int RYS_NINT = 60;
constexpr int RYS_DEG = 12;
constexpr int RYS_NCOEF = RYS_DEG + 1;
constexpr double RYS_TMAX = 60.0;
// table layout: for n = 1..5 roots, RYS_NINT intervals x 2n functions (n roots
// then n weights) x RYS_NCOEF coefficients; then per n the large-T limit:
// MAXROOT Gauss-Hermite r_i (u = r_i/T) followed by MAXROOT W_i (w = W_i/sqrt T)
__host__ __device__ constexpr int rys_table_off(int n) { return RYS_NINT * RYS_NCOEF * n * (n - 1); }
__host__ __device__ constexpr int rys_herm_off(int n) {
    return rys_table_off(MAXROOT + 1) + (n - 1) * 2 * MAXROOT;
}
constexpr int RYS_TABLE_SIZE = rys_herm_off(MAXROOT + 1);

enum PairClass { SS = 0, SP, PP, SD, PD, DD, NPC };
enum Op { OP_GE = 0, OP_GT = 1, OP_NONE = 2 };
enum Tile { TILE_SQRT = 0, TILE_E9 = 1, TILE_E8 = 2, TILE_NONE = 3 };

// One reference kernel (intABCD) and its screening / digestion behaviour.
struct KernelDesc {
    const char *name;
    int bra, ket;        // pair classes
    bool tri;            // same-class triangle (kkll <= iijj)
    bool rys;            // generated Rys kernel (else rotated-axis)
    bool cross;          // pre-screen against the other class's maximum
    int op;              // product test: >=, > or none
    int tile;            // tile size used by the rank split
    bool ketmajor;       // flat index runs bra-fastest (Rys product kernels)
    bool digest_schwarz; // digestion skip uses cutoff_schwarz (else eri_cut)
    double asym;         // asymptotic-root threshold (rot: T > 25; Rys: T >= x)
    int la, lb, lc, ld;  // shell angular momenta in the engine's orientation
};
extern const KernelDesc KDESC[NKERN];

// Device views ----------------------------------------------------------------
struct DevBasis {
    const double4 *shell_xyz;  // per shell: x, y, z, -
    const int *shell_bf0;      // per shell: 0-based first basis function
    const int2 *pair_shell;    // per global pair: (A, B), L_A >= L_B
    const int *pair_prim0;     // first primitive pair
    const int *pair_nprim;     // number of kept primitive pairs
    const double4 *prim_P;     // Px, Py, Pz, p
    const double *prim_K;      // sqrt(2 pi^2.5) c_a c_b exp(-mu R^2) / p
};

struct DevPlan {
    int nbra, nket;
    const int *bra_ids, *ket_ids;    // global pair ids, sorted by xint desc
    const int *bra_orig, *ket_orig;  // positions in the reference's compacted lists
    const long long *pref;           // nbra+1 exclusive prefix of work items
    long long total;
    // fp32 split: items [pref[i], pref[i]+n64[i]) of bra i are FP64, the rest
    // FP32.  n64 == nullptr means everything is FP64.
    const int *split;                // per bra: first FP32 ket position
};

struct RankSplit {
    int rank, nsize;       // nsize == 1 -> no filtering
    int tile;
    long long ntot;        // reference iteration count of the kernel
    int nbra_ref, nket_ref;
    int tri, ketmajor;
};

// Host state -------------------------------------------------------------------
struct PlanHost {
    int nbra = 0, nket = 0;
    std::vector<int> bra_ids, ket_ids, bra_orig, ket_orig, ncount;
    std::vector<double> bra_x, ket_x;
    std::vector<long long> pref;
    long long total = 0;
    long long ntot_ref = 0;  // reference iteration count (rank split)
    int nbra_ref = 0, nket_ref = 0;
    // device copies
    int *d_bra = nullptr, *d_ket = nullptr, *d_bra_orig = nullptr, *d_ket_orig = nullptr;
    long long *d_pref = nullptr;
    double *d_bra_x = nullptr, *d_ket_x = nullptr;
    int *d_ncount = nullptr;
    // mixed precision: per build
    long long *d_pref64 = nullptr, *d_pref32 = nullptr;
    int *d_split = nullptr;
    long long total64 = 0, total32 = 0;
};

struct BasisHost {
    int nsh = 0, natoms = 0, num_bas = 0, mxgtot = 0;
    std::vector<int> ang_mom, contr_num, sh_loc, atom_num, atom_loc, start_bas, end_bas;
    std::vector<double> exponents, cs, cp, cd, cf, coords, schwrz;
};

struct PairsHost {
    // global pair numbering: class offsets
    int class_off[NPC + 1] = {0};
    std::vector<int> ish, jsh;    // reference order (first, second)
    std::vector<double> xint;
    std::vector<int2> shell;      // engine orientation
    std::vector<int> prim0, nprim;
    std::vector<double4> P;
    std::vector<double> K;
    int nl[3] = {0, 0, 0};
};

struct DeviceBuffers {
    double4 *shell_xyz = nullptr;
    int *shell_bf0 = nullptr;
    int2 *pair_shell = nullptr;
    int *pair_prim0 = nullptr, *pair_nprim = nullptr;
    double4 *prim_P = nullptr;
    double *prim_K = nullptr;
    double *D = nullptr, *F = nullptr;
    long long *scratch_total = nullptr;  // device counters (mixed split)
    size_t bytes = 0;
};

// Rys root/weight tables (host generated once, uploaded per handle), layout above
const std::vector<double> &rys_table_host();

// Launchers (kernels.cu) ------------------------------------------------------
struct LaunchCtx {
    DevBasis basis;
    const double *rys_tab;
    const double *D;
    double *F;
    double schwarz_cut, eri_cut;
    cudaStream_t stream;
    int num_sms;
};

cudaError_t launch_class(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs,
                         int precision);  // precision 0: fp64 items, 1: fp32 items
cudaError_t launch_maxabs(const double *x, long long n, unsigned long long *out,
                          cudaStream_t stream);
cudaError_t launch_split(int nbra, const double *bra_x, const double *ket_x, const int *ncount,
                         const unsigned long long *maxd, double fp32_cut, int *split,
                         long long *pref64, long long *pref32, cudaStream_t stream);
cudaError_t launch_schwarz(int pair_class, int npairs, int pair_off, const DevBasis &b,
                           const double *rys_tab, double *out_per_pair, cudaStream_t stream);

}  // namespace liberi
