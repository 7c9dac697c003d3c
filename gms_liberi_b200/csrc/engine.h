// engine.h -- internal structures of the B200 Fock-build engine.
//
// Host side (host.cpp) builds, once per geometry, the device-resident shell,
// pair and quartet-plan buffers described here; the device side (kernels.cu)
// evaluates the 21 s/p/d quartet classes of the reference driver
// (src/liberi_driver.F90:69-102) and the 34 classes of its f block
// (src/liberi_driver.F90:103-160) with Rys quadrature and digests them into
// the packed Fock matrix.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace liberi {

constexpr int NKERN = 21;     // s/p/d classes: per-class kernels, FP32 tier, batching, tuning
constexpr int NKERN_F = 34;   // f classes: one shared-memory kernel, FP64
constexpr int NKALL = NKERN + NKERN_F;
constexpr int NVARIANT = 3;  // kernel shape variants per class and precision
constexpr int MAXROOT = 5;
// Rys tables: intervals of width 1/4 in T on [0, RYS_TMAX), degree-7 power
// basis in x = 2(4T - k) - 1 (8 coefficients: four aligned double2 loads per
// function; interpolation error below 6e-15 relative for 1..5 roots).
constexpr int RYS_PER_UNIT = 4;
constexpr int RYS_NINT = 60 * RYS_PER_UNIT;
constexpr int RYS_DEG = 7;
constexpr int RYS_NCOEF = 8;
constexpr double RYS_TMAX = 60.0;
// table layout: for n = 1..5 roots, RYS_NINT intervals x 2n functions (n roots
// then n weights) x RYS_NCOEF coefficients; then per n the large-T limit:
// MAXROOT Gauss-Hermite r_i (u = r_i/T) followed by MAXROOT W_i (w = W_i/sqrt T)
__host__ __device__ constexpr int rys_table_off(int n) { return RYS_NINT * RYS_NCOEF * n * (n - 1); }
__host__ __device__ constexpr int rys_herm_off(int n) {
    return rys_table_off(MAXROOT + 1) + (n - 1) * 2 * MAXROOT;
}
constexpr int RYS_TABLE_SIZE = rys_herm_off(MAXROOT + 1);
// Single-precision tables for the FP32 tier: intervals of width 1/8 on
// [0, RYS_TMAX), degree-3 power basis in x = 2(8T - k) - 1 (4 coefficients:
// two functions per 256-bit load; interpolation error below 5e-8 relative);
// then the large-T limit as above, in float.
constexpr int RYSF_PER_UNIT = 8;
constexpr int RYSF_NINT = 60 * RYSF_PER_UNIT;
constexpr int RYSF_DEG = 3;
constexpr int RYSF_NCOEF = 4;
__host__ __device__ constexpr int rysf_table_off(int n) { return RYSF_NINT * RYSF_NCOEF * n * (n - 1); }
__host__ __device__ constexpr int rysf_herm_off(int n) {
    return rysf_table_off(MAXROOT + 1) + (n - 1) * 2 * MAXROOT;
}
constexpr int RYSF_TABLE_SIZE = rysf_herm_off(MAXROOT + 1);
// Tables of the f classes: 1..7 roots on [0, RYS7_TMAX) (the 7-root classes
// switch to the large-T limit at 65), same interval width and degree as above;
// then per n the large-T limit: MAXROOT7 r_i followed by MAXROOT7 W_i.
constexpr int MAXROOT7 = 7;
constexpr double RYS7_TMAX = 65.0;
constexpr int RYS7_NINT = 65 * RYS_PER_UNIT;
__host__ __device__ constexpr int rys7_table_off(int n) { return RYS7_NINT * RYS_NCOEF * n * (n - 1); }
__host__ __device__ constexpr int rys7_herm_off(int n) {
    return rys7_table_off(MAXROOT7 + 1) + (n - 1) * 2 * MAXROOT7;
}
constexpr int RYS7_TABLE_SIZE = rys7_herm_off(MAXROOT7 + 1);

// the six s/p/d pair classes, then the f ones (lower-L shell first in the
// reference order, src/liberi_shell_pair.F90:1285-1682)
enum PairClass { SS = 0, SP, PP, SD, PD, DD, SF, PF, DF, FF, NPC };
constexpr int NPC_SPD = 6;
enum Op { OP_GE = 0, OP_GT = 1, OP_NONE = 2 };
enum Tile { TILE_SQRT = 0, TILE_E9 = 1, TILE_E8 = 2, TILE_NONE = 3 };

// One reference kernel (intABCD) and its screening / digestion behaviour.
struct KernelDesc {
    const char *name;
    int bra, ket;        // reference pair classes (bra, ket)
    bool tri;            // same-class triangle (kkll <= iijj)
    bool rys;            // generated Rys kernel (else rotated-axis)
    bool cross;          // pre-screen against the other class's maximum
    int op;              // product test: >=, > or none
    int tile;            // tile size used by the rank split
    bool ketmajor;       // flat index runs bra-fastest (Rys product kernels)
    bool digest_schwarz; // digestion skip uses cutoff_schwarz (else eri_cut)
    double asym;         // asymptotic-root threshold (rot: T > 25; Rys: T >= x)
    bool swap;           // engine rows = the reference's ket class (larger block)
    int la, lb, lc, ld;  // engine orientation: rows (A,B), kets (C,D), L_A >= L_B
};
extern const KernelDesc KDESC[NKALL];

// Device views ----------------------------------------------------------------
struct DevBasis {
    const double4 *shell_xyz;  // per shell: x, y, z, -
    const int *shell_bf0;      // per shell: 0-based first basis function
    const int2 *pair_shell;    // per global pair: (A, B), L_A >= L_B
    const int *pair_prim0;     // first primitive pair
    const int *pair_nprim;     // number of kept primitive pairs
    const double4 *prim_P;     // Px, Py, Pz, p
    const double2 *prim_X;     // sqrt(2 pi^2.5) c_a c_b exp(-mu R^2) / p, 0.5 / p
    const float4 *prim_PAf;    // FP32 tier, two float4 per primitive pair (one 256-bit load):
                               // (Px, Py, Pz, p), (P - A rounded once from FP64, prefactor)
    const float *prim_bound;   // per primitive pair sqrt(max |(ab|ab)|) of that primitive alone
                               // (the FP32 tier's primitive screening), or null
};

// One launch of a class: a list of CTA tasks (bra position, first ket
// position, ket count) over the plan's sorted lists.
// Batched launches: one task list over several molecules; task.w selects the
// molecule, whose device data and class lists come from these views.
struct MolView {
    DevBasis b;
    const double *D;  // packed density (caller's buffer)
    double *Dsq;      // this iteration's D as a full nbf x nbf matrix (batch-owned)
    double *F;
    float *Df;  // FP32 tier of a mixed-precision batch: the full D in float
    int nbf;
    int pad;
};
struct ClassView {
    const int *bra_ids, *ket_ids;
    const double *bra_x, *ket_x;  // Schwarz values of the lists (mixed-precision split)
    const double4 *ket_rec;       // ket records of the list (two double4 per position)
};

// Per ket position of a class plan, what a quartet needs of its ket pair (C,D)
// in two 256-bit loads that are contiguous across the lanes of a warp:
//   [0] = (C-D x, y, z, C.x), [1] = (C.y, C.z, bits of first functions
//   bf0(C) | bf0(D) << 32, bits of first primitive pair | kept count << 32).
constexpr int KET_REC = 2;

struct DevPlan {
    const int *bra_ids, *ket_ids;    // global pair ids, sorted by xint desc
    const double4 *ket_rec;          // ket records (KET_REC double4 per ket position)
    const int *bra_orig, *ket_orig;  // positions in the reference's compacted lists
    const int4 *tasks;
    const int *ntasks_dev;           // task count on the device (per-build lists) or null
    int ntasks;                      // static count, or capacity for per-build lists
    bool swapped;
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
    std::vector<int4> items;  // (bra position, ket segment start, surviving count, -)
    std::vector<double> bra_x, ket_x;
    std::vector<long long> pref;
    long long total = 0;
    long long ntot_ref = 0;  // reference iteration count (rank split)
    int nbra_ref = 0, nket_ref = 0;
    int chunk = 512;         // kets per CTA task
    std::vector<int4> tasks; // static FP64 task list
    int task_cap = 0;        // capacity of the per-build (mixed) lists
    // device copies
    int *d_bra = nullptr, *d_ket = nullptr, *d_bra_orig = nullptr, *d_ket_orig = nullptr;
    double *d_bra_x = nullptr, *d_ket_x = nullptr;
    double4 *d_ket_rec = nullptr;
    int4 *d_items = nullptr;
    int4 *d_tasks = nullptr;
    // mixed precision: per-build task lists
    int4 *d_tasks64 = nullptr, *d_tasks32 = nullptr;
    int *d_ntasks = nullptr;  // [0] fp64 count, [1] fp32 count, [2] fp32 quartets (lo), [3] (hi)
};

struct BasisHost {
    int nsh = 0, natoms = 0, num_bas = 0, mxgtot = 0;
    std::vector<int> ang_mom, contr_num, sh_loc, atom_num, atom_loc, start_bas, end_bas;
    std::vector<double> exponents, cs, cp, cd, cf, coords, schwrz;
};
constexpr int MAXL = 3;  // f

struct PairsHost {
    // global pair numbering: class offsets
    int class_off[NPC + 1] = {0};
    std::vector<int> ish, jsh;    // reference order (first, second)
    std::vector<double> xint;
    std::vector<int2> shell;      // engine orientation
    std::vector<int> prim0, nprim;
    std::vector<int> kab;         // contraction-pattern key K_a * K_b
    std::vector<double4> P;
    std::vector<double2> X;
    int nl[MAXL + 1] = {0, 0, 0, 0};
};

struct DeviceBuffers {
    double4 *shell_xyz = nullptr;
    int *shell_bf0 = nullptr;
    int2 *pair_shell = nullptr;
    int *pair_prim0 = nullptr, *pair_nprim = nullptr;
    double4 *prim_P = nullptr;
    double2 *prim_X = nullptr;
    float4 *prim_PAf = nullptr;
    float *prim_bound = nullptr;
    double *D = nullptr, *F = nullptr;
    double *Dsq = nullptr;  // the build's D as a full n x n matrix (class kernels read it)
    float *Df = nullptr;    // FP32 tier: the same in single precision
    // open-shell builds (made at the first one): the Coulomb and exchange
    // densities as two consecutive full n x n matrices, and their float copies
    double *uhf_sq = nullptr;
    float *uhf_sqf = nullptr;
    long long *scratch_total = nullptr;  // device counters (mixed split)
    size_t bytes = 0;
};

// Rys root/weight tables (host generated once, uploaded per handle), layout above
const std::vector<double> &rys_table_host();
const std::vector<float> &rys_table_f32_host();
const std::vector<double> &rys_table7_host();  // the f classes' table (1..7 roots)

// Launchers (kernels.cu) ------------------------------------------------------
// builds of at most FAN_MAX_QUARTETS screened quartets spread their classes
// over FAN_STREAMS streams (option "overlap")
constexpr int FAN_STREAMS = 8;
constexpr long long FAN_MAX_QUARTETS = 25000000;

struct LaunchCtx {
    DevBasis basis;
    const double *rys_tab;
    const float *rys_tabf;
    const double *D;
    const float *Df;
    double *F;
    double schwarz_cut, eri_cut;
    cudaStream_t stream;
    int num_sms;
    // FP32 tier: max|D| of the build (ordered bits; per molecule for batches)
    // and the primitive screening cut (fp32_prim * fp32_cut; 0 = off)
    const unsigned long long *maxd = nullptr;
    double prim_cut = 0.0;
    // open-shell builds: the exchange terms read a second full matrix at D + k_offset (0 = D itself)
    size_t k_offset = 0;
    const double *rys_tab7 = nullptr;  // f classes: the 1..7-root table
};

cudaError_t launch_class(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs,
                         int precision, int nbf, int tile_rows, int variant);  // precision 0: FP64, 1: FP32
// f class k (NKERN <= k < NKALL), FP64: one CTA per task, the task's
// quartets in turn, every quartet evaluated and digested by the whole CTA
cudaError_t launch_fclass(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs, int nbf);
// adds {count, sum, xor} of the hashes of the quartets a launch of class k over
// this plan's task list would evaluate to out[0..2] (zeroed by the caller)
cudaError_t launch_quartet_fp(int k, const LaunchCtx &ctx, const DevPlan &plan, const RankSplit &rs,
                              unsigned long long *out);
// one launch of class k over the tasks of several molecules (task.w = molecule)
cudaError_t launch_class_batch(int k, const LaunchCtx &ctx, const int4 *tasks, int ntasks, int nbf_max,
                               const MolView *d_mols, const ClassView *d_cviews, bool swapped, int precision,
                               const int *ntasks_dev);
cudaError_t launch_zero_fock(const MolView *d_mols, int nmol, long long max_ntri, cudaStream_t stream);
// batch: every molecule's D as a full matrix (Dsq), and for a mixed-precision
// batch its float copy (Df) and max|D| (as ordered bits, maxd non-null)
cudaError_t launch_batch_prep(const MolView *d_mols, int nmol, long long max_nsq, unsigned long long *maxd,
                              cudaStream_t stream);
// mixed-precision batch: FP64/FP32 task lists of one class over every molecule's items
// (item.w = molecule), as split_tasks_kernel does for one molecule
cudaError_t launch_split_batch(int nitems, const int4 *items, const ClassView *d_cviews,
                               const unsigned long long *maxd, double fp32_cut, int chunk, int4 *tasks64,
                               int4 *tasks32, int *counts, cudaStream_t stream);
// full n x n copy of a packed density, and its float copy when sqf is non-null
cudaError_t launch_unpack(const double *packed, int n, double *sq, float *sqf, cudaStream_t st);
// open-shell builds: sq = ca * A + cb * B from two packed matrices (full n x n, float copy when sqf)
cudaError_t launch_unpack_combo(const double *pa, const double *pb, double ca, double cb, int n, double *sq,
                                float *sqf, cudaStream_t st);
cudaError_t launch_maxabs(const double *x, long long n, unsigned long long *out,
                          cudaStream_t stream);
cudaError_t launch_split_tasks(int nitems, const int4 *items, const double *bra_x, const double *ket_x,
                               const unsigned long long *maxd, double fp32_cut, int chunk,
                               int4 *tasks64, int4 *tasks32, int *counts, cudaStream_t stream);
// Schwarz values of the f pair classes (sf, pf, df, ff) with the f classes'
// shared-memory evaluation and the 1..7-root table (k_f.cu)
cudaError_t launch_fschwarz(int pair_class, int npairs, int pair_off, const DevBasis &b, const double *rys_tab7,
                            double *out, cudaStream_t stream);
cudaError_t launch_schwarz(int pair_class, int npairs, int pair_off, const DevBasis &b,
                           const double *rys_tab, double *out_per_pair, cudaStream_t stream);
// per primitive pair of one pair class: sqrt(max |(ab|ab)|) of the primitive alone, rounded up to float
cudaError_t launch_prim_bound(int pair_class, int npairs, int pair_off, const DevBasis &b, const double *rys_tab,
                              float *out_per_prim, cudaStream_t stream);

// host-side inputs of the Schwarz generator (host.cpp) and the thread's
// last-error message, for the allocation-free entry point (noalloc.cu)
int schwarz_host_inputs(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot, const int32_t *ang_mom,
                        const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                        const int32_t *atom_loc, const double *exponents, const double *contr_coef_s,
                        const double *contr_coef_p, const double *contr_coef_d, const double *coords,
                        BasisHost &basis, PairsHost &pairs, std::vector<double4> &shell_xyz);
int set_error(int code, const char *msg);
// the CUDA device of an NCCL communicator (comm.cpp), -1 for none
int comm_device(struct liberi_comm_s *comm);

}  // namespace liberi
