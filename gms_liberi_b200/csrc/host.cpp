// host.cpp -- C ABI, setup and quartet planning of the B200 Fock-build engine.
//
// Mirrors libERI's handle API (src/interface/liberi_interface.F90) and GAMESS
// wrapper (src/interface/gms_liberi_wrapper.F90).  Setup restates the
// reference's shell classification and pair classes
// (src/liberi_shell_pair.F90:39-1283) and its per-kernel screening
// (src/rhf/rot_axis/int*.F90 headers), then stores a device-resident plan per
// kernel class: bra pairs sorted by Schwarz value, for each bra the number of
// surviving kets, which form a prefix of the Schwarz-sorted ket list.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <system_error>
#include <thread>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/liberi_b200.h"
#include "engine.h"

namespace liberi {

// Driver order and per-kernel screening (src/liberi_driver.F90:69-102):
// pre-screen (cross: int0001.F90:67-84; own: int2211_rysgen.F90:295-310),
// product operator (int0000.F90:106-107 ">=", int0001.F90:120-121 ">",
// int2222_rysgen.F90:428-436 none), tiles (int0000.F90:76-81 sqrt(3.75e9),
// int0001.F90:90 3.75e9, int0002.F90:84 3.75e8), flat order
// (int0001.F90:117 bra-major, int2211_rysgen.F90:351 bra-fastest), digestion
// cut (cutoff_schwarz int0000.F90:246, literal 5e-11 int0002.F90:403) and
// asymptotic thresholds (t_max=25, Rys 43/49/55).
// Engine orientation: the "rows" pair (A,B) is the class with the larger
// Cartesian block (its rows of F are staged in shared memory), the kets (C,D)
// the smaller; `swap` marks classes whose rows are the reference's ket list.
const KernelDesc KDESC[NKALL] = {
    //  name      bra ket  tri    rys    cross  op      tile       kmaj   dsch   asym  swap   la lb lc ld
    {"int0000", SS, SS, true, false, false, OP_GE, TILE_SQRT, false, true, 25.0, false, 0, 0, 0, 0},
    {"int0001", SS, SP, false, false, true, OP_GT, TILE_E9, false, true, 25.0, true, 1, 0, 0, 0},
    {"int0011", SS, PP, false, false, true, OP_GT, TILE_E9, false, true, 25.0, true, 1, 1, 0, 0},
    {"int0111", SP, PP, false, false, true, OP_GT, TILE_E9, false, false, 25.0, true, 1, 1, 1, 0},
    {"int0101", SP, SP, true, false, false, OP_GE, TILE_NONE, false, false, 25.0, false, 1, 0, 1, 0},
    {"int1111", PP, PP, true, false, false, OP_GE, TILE_NONE, false, true, 25.0, false, 1, 1, 1, 1},
    {"int0002", SS, SD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, true, 2, 0, 0, 0},
    {"int0012", SS, PD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, true, 2, 1, 0, 0},
    {"int0102", SP, SD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, true, 2, 0, 1, 0},
    {"int0112", SP, PD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, true, 2, 1, 1, 0},
    {"int0022", SS, DD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, true, 2, 2, 0, 0},
    {"int0122", SP, DD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, true, 2, 2, 1, 0},
    {"int1102", PP, SD, false, false, true, OP_GT, TILE_E8, false, false, 25.0, false, 1, 1, 2, 0},
    {"int0202", SD, SD, true, false, false, OP_GT, TILE_NONE, false, false, 25.0, false, 2, 0, 2, 0},
    {"int2211", DD, PP, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 2, 2, 1, 1},
    {"int2121", PD, PD, true, true, false, OP_GT, TILE_NONE, false, false, 49.0, false, 2, 1, 2, 1},
    {"int2120", PD, SD, false, true, false, OP_GT, TILE_E8, true, false, 43.0, false, 2, 1, 2, 0},
    {"int2111", PD, PP, false, true, false, OP_GT, TILE_E8, true, false, 43.0, false, 2, 1, 1, 1},
    {"int2220", DD, SD, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 2, 2, 2, 0},
    {"int2221", DD, PD, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 2, 2, 2, 1},
    {"int2222", DD, DD, true, true, false, OP_NONE, TILE_NONE, false, false, 55.0, false, 2, 2, 2, 2},
    // the f block (liberi_driver.F90:103-160): own-class pre-screens, ">"
    // product test except int3333 (none), 3.75e8 tiles for the product
    // kernels, bra-fastest flat order in the Rys product kernels and
    // bra-major in the ERIC ones (int0030_ericgen.F90:66-124,
    // int3011_rysgen.F90:213-274, int3333_rysgen.F90:829-867); digestion at
    // 5e-11; the ERIC kernels (rys false) take the Boys-function rule with the
    // large-T form above t_max = 25, the Rys ones switch at 43/49/55/60/65
    // for 3..7 roots.  The rows are the reference's bra list (no swap).
    {"int3333", FF, FF, true, true, false, OP_NONE, TILE_NONE, false, false, 65.0, false, 3, 3, 3, 3},
    {"int0030", SS, SF, false, false, false, OP_GT, TILE_E8, false, false, 25.0, false, 0, 0, 3, 0},
    {"int0031", SS, PF, false, false, false, OP_GT, TILE_E8, false, false, 25.0, false, 0, 0, 3, 1},
    {"int0032", SS, DF, false, false, false, OP_GT, TILE_E8, false, false, 25.0, false, 0, 0, 3, 2},
    {"int1030", SP, SF, false, false, false, OP_GT, TILE_E8, false, false, 25.0, false, 1, 0, 3, 0},
    {"int3330", FF, SF, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 3, 3, 0},
    {"int3011", SF, PP, false, true, false, OP_GT, TILE_E8, true, false, 43.0, false, 3, 0, 1, 1},
    {"int3020", SF, SD, false, true, false, OP_GT, TILE_E8, true, false, 43.0, false, 3, 0, 2, 0},
    {"int2130", PD, SF, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 2, 1, 3, 0},
    {"int2230", DD, SF, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 2, 2, 3, 0},
    {"int3030", SF, SF, true, true, false, OP_GT, TILE_NONE, false, false, 49.0, false, 3, 0, 3, 0},
    {"int3110", PF, SP, false, true, false, OP_GT, TILE_E8, true, false, 43.0, false, 3, 1, 1, 0},
    {"int3111", PF, PP, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 1, 1, 1},
    {"int3120", PF, SD, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 1, 2, 0},
    {"int3121", PF, PD, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 1, 2, 1},
    {"int2231", DD, PF, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 2, 2, 3, 1},
    {"int3130", PF, SF, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 1, 3, 0},
    {"int3131", PF, PF, true, true, false, OP_GT, TILE_NONE, false, false, 55.0, false, 3, 1, 3, 1},
    {"int3210", DF, SP, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 2, 1, 0},
    {"int3331", FF, PF, false, true, false, OP_GT, TILE_E8, true, false, 60.0, false, 3, 3, 3, 1},
    {"int3211", DF, PP, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 2, 1, 1},
    {"int3220", DF, SD, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 2, 2, 0},
    {"int3221", DF, PD, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 2, 2, 1},
    {"int3222", DF, DD, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 2, 2, 2},
    {"int3230", DF, SF, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 2, 3, 0},
    {"int3231", DF, PF, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 2, 3, 1},
    {"int3232", DF, DF, true, true, false, OP_GT, TILE_NONE, false, false, 60.0, false, 3, 2, 3, 2},
    {"int3300", FF, SS, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 3, 0, 0},
    {"int3310", FF, SP, false, true, false, OP_GT, TILE_E8, true, false, 49.0, false, 3, 3, 1, 0},
    {"int3311", FF, PP, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 3, 1, 1},
    {"int3320", FF, SD, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 3, 2, 0},
    {"int3321", FF, PD, false, true, false, OP_GT, TILE_E8, true, false, 55.0, false, 3, 3, 2, 1},
    {"int3322", FF, DD, false, true, false, OP_GT, TILE_E8, true, false, 60.0, false, 3, 3, 2, 2},
    {"int3332", FF, DF, false, true, false, OP_GT, TILE_E8, true, false, 60.0, false, 3, 3, 3, 2},
};

static const int PC_L1[NPC] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 3};  // reference pair order (first, second)
static const int PC_L2[NPC] = {0, 1, 1, 2, 2, 2, 3, 3, 3, 3};
static const double CUX = 50.0;                    // src/liberi_parameters.F90:44
static const double SQRT_TWOPI52 = 5.9149671727956128778;  // sqrt(2 pi^(5/2))
static const size_t TILE_MAX_BYTES = 160 * 1024;            // shared-memory F rows per CTA
static const int CLASS_CTA_THREADS = 128;
static const int TUNE_CHUNKS[] = {128, 256, 512, 1024, 2048};  // kets per CTA task the autotuner tries

static int ncart_l(int l) { return (l + 1) * (l + 2) / 2; }

// default kets per CTA task (the autotuner may override per s/p/d class; an f
// class CTA evaluates its task's quartets one after another)
static int default_chunk(int k) {
    const KernelDesc &d = KDESC[k];
    const int nc = ncart_l(d.la) * ncart_l(d.lb) * ncart_l(d.lc) * ncart_l(d.ld);
    if (k >= NKERN) return 1;  // an f quartet is a group's work: one ket per task keeps every SM busy
    // (ss|dd) and (sp|dd): few kets per row pair survive the screening; short
    // tasks spread them (C60: 0.35 -> 0.32 and 1.12 -> 1.08 ms)
    if (k == 10 || k == 11) return CLASS_CTA_THREADS;
    // measured on C60 (FP64, liberi_c_autotune): longer tasks for the low-L
    // classes ((sp|sp) 13.00 -> 12.67 ms at 2048 kets, (ss|sp) 10.41 -> 10.32,
    // (ss|pp) 5.93 -> 5.84, (pp|pp) 9.61 -> 9.53 at 1024), shorter ones for
    // (sd|sd) (0.70 -> 0.68 ms at 128) and (pd|pd) (4.30 -> 4.25 ms at 256)
    switch (k) {
        case 1: case 4: return 2048;
        case 2: case 3: case 5: return 1024;
        case 13: return 128;
        case 15: return 256;
        default: break;
    }
    const int qpt = nc >= 216 ? 1 : (nc >= 54 ? 2 : 4);
    return CLASS_CTA_THREADS * qpt;
}

}  // namespace liberi

using namespace liberi;

// ---- error handling -------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? LIBERI_E_NOMEM : LIBERI_E_DEVICE, \
                        "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// Makes `dev` current for one C-ABI call and restores the caller's current
// device on return (a library must not move its caller's CUDA context).
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

// A non-blocking stream at the device's greatest priority.
static cudaError_t high_priority_stream(cudaStream_t *st) {
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e != cudaSuccess) return e;
    return cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, greatest);
}

// ---- handle ------------------------------------------------------------------------
struct liberi_handle_s {
    // options (defaults reproduce the reference constants)
    double schwarz_cut = 5.00000000000000018e-11;  // liberi_parameters.F90:38
    double eri_cut = 5.0e-11;
    double fp32_cut = 1.0e-7;
    // FP32 tier: primitive quartets with bound * max|D| below fp32_prim * fp32_cut are skipped
    double fp32_prim = 1.0e-8;
    // device bytes a setup may take (0: no limit); checked on the host before any device work
    double max_device_bytes = 0.0;
    int precision = 0;
    int device = 0;
    uint32_t class_mask = (1u << NKERN) - 1;
    int rank_split = 0;  // 0: the reference's per-kernel split, 1: cost-balanced contiguous slices
    // classes allowed to stage F rows in shared memory: none by default (the
    // tile's shared memory costs more L1, where tables and spills live, than
    // its atomics save; measured on C60 and the batched molecules)
    uint32_t tile_mask = 0;
    // FP64 builds: classes launched on the side stream beside the others: the
    // high-L classes of few long CTAs and the small low-occupancy ones
    // ((ss|dd), (sp|dd), (sd|sd) and the seven Rys classes).  Measured on C60:
    // 100.40 ms with (dd|dd) and (dd|pd) alone there, 99.37 ms with these ten
    // (99.60 without (pd|sd) and (pd|pp), 99.51 with (pp|sd) added).
    uint32_t side_mask = (1u << 10) | (1u << 11) | (1u << 13) | (1u << 14) | (1u << 15) | (1u << 16) | (1u << 17) |
                         (1u << 18) | (1u << 19) | (1u << 20);
    int chunk[NKALL] = {};  // kets per CTA task per class (0 = default)
    int variant[2][NKERN] = {};  // kernel shape variant per class, FP64 / FP32 tier
    bool timing = false;
    bool last_split_lists = false;  // the last build ran the per-build FP64/FP32 task lists
    cudaEvent_t ev[NKERN + 1][2] = {};
    bool ev_recorded[NKERN] = {};
    bool plan_dirty = false;

    bool initialized = false;
    int my_rank = 0, num_procs = 1;
    BasisHost basis;
    PairsHost pairs;
    PlanHost plan[NKALL];
    long long fq[NKERN_F] = {}, fprim[NKERN_F] = {};  // per f class: quartets, primitive quartets
    DeviceBuffers dev;
    double *d_tab = nullptr;
    double *d_tab7 = nullptr;  // the f classes' 1..7-root table (bases with f shells)
    float *d_tabf = nullptr;
    unsigned long long *d_maxd = nullptr;
    cudaStream_t stream = nullptr;
    // mixed builds run their FP64 task lists on a second stream beside the
    // FP32 lists, FP64 builds the classes of side_mask (forked from and joined
    // back into the build's stream)
    bool overlap = true;
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // small builds spread their classes over FAN_STREAMS streams (option "fan")
    bool fan_out = true;
    cudaStream_t fan[FAN_STREAMS] = {};
    cudaEvent_t fan_ev[FAN_STREAMS] = {};
    int num_sms = 148;
    liberi_stats stats;
    std::vector<void *> allocs;
    // one allocation each for the basis data and for the class plans, carved
    // into the handle's buffers (arena: the one being carved, or null)
    struct Arena {
        char *base = nullptr;
        size_t size = 0, used = 0;
    } arena_basis, arena_plans, *arena = nullptr;
};

// Handle buffers are carved from one stream-ordered allocation per group
// (basis data, class plans) at DEV_ALIGN-byte offsets: a few hundred small
// cudaMallocAsync calls per handle made the allocator's bookkeeping, and so
// every further setup, grow with the number of live handles.
constexpr size_t DEV_ALIGN = 256;
static size_t dev_round(size_t bytes) { return (bytes + DEV_ALIGN - 1) & ~(DEV_ALIGN - 1); }
// bytes one dev_upload of n elements takes (none for n == 0), and one dev_alloc
static size_t up_bytes(size_t n, size_t elem) { return n ? dev_round(n * elem) : 0; }
static size_t al_bytes(size_t n, size_t elem) { return dev_round((n ? n : 1) * elem); }

static cudaError_t dev_get(liberi_handle h, size_t bytes, void **p) {
    bytes = dev_round(bytes);
    if (h->arena) {
        if (h->arena->used + bytes > h->arena->size) return cudaErrorMemoryAllocation;  // accounting mismatch
        *p = h->arena->base + h->arena->used;
        h->arena->used += bytes;
    } else {
        cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
        if (e != cudaSuccess) return e;
        h->allocs.push_back(*p);
    }
    h->dev.bytes += bytes;
    return cudaSuccess;
}

// opens an arena of exactly `bytes` for the uploads of one group
static cudaError_t arena_open(liberi_handle h, liberi_handle_s::Arena &a, size_t bytes) {
    a = liberi_handle_s::Arena();
    if (bytes) {
        void *p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, bytes, h->stream);
        if (e != cudaSuccess) return e;
        h->allocs.push_back(p);
        a.base = static_cast<char *>(p);
        a.size = bytes;
    }
    h->arena = &a;
    return cudaSuccess;
}
struct ArenaScope {  // stops carving when the group's uploads end, on every path
    liberi_handle h;
    ~ArenaScope() { h->arena = nullptr; }
};

// Handle memory is stream-ordered on the handle's stream (cudaMallocAsync /
// cudaFreeAsync), so setting up or releasing one handle never synchronises
// the device and stalls builds of other handles in flight.  Allocation sites
// synchronise the handle's stream before the memory is used on other
// streams; releases require the caller's builds on its own streams to have
// completed (liberi_c_fock_build_device).  The host source of an upload may
// be released on return (pageable copies are staged before the call returns).
template <typename T>
static cudaError_t dev_upload(liberi_handle h, T **dst, const T *src, size_t n) {
    *dst = nullptr;
    if (n == 0) return cudaSuccess;
    cudaError_t e = dev_get(h, n * sizeof(T), (void **)dst);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, h->stream);
}

template <typename T>
static cudaError_t dev_alloc(liberi_handle h, T **dst, size_t n) {
    *dst = nullptr;
    if (n == 0) n = 1;
    return dev_get(h, n * sizeof(T), (void **)dst);
}

// frees an allocation of its own (not a piece carved from an arena)
static void dev_release(liberi_handle h, void *p) {
    auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
    if (it == h->allocs.end()) return;
    cudaFreeAsync(p, h->stream);
    h->allocs.erase(it);
}

static void free_device(liberi_handle h) {
    for (void *p : h->allocs) cudaFreeAsync(p, h->stream);
    h->allocs.clear();
    h->arena_basis = h->arena_plans = liberi_handle_s::Arena();
    h->arena = nullptr;
    h->dev = DeviceBuffers();
    h->d_tab = nullptr;
    h->d_tab7 = nullptr;
    h->d_tabf = nullptr;
    h->d_maxd = nullptr;
    for (int k = 0; k < NKALL; k++) h->plan[k] = PlanHost();
    if (h->stream) {
        cudaStreamDestroy(h->stream);
        h->stream = nullptr;
    }
    if (h->side) cudaStreamDestroy(h->side);
    if (h->fork_ev) cudaEventDestroy(h->fork_ev);
    if (h->join_ev) cudaEventDestroy(h->join_ev);
    h->side = nullptr;
    h->fork_ev = h->join_ev = nullptr;
    for (int i = 0; i < FAN_STREAMS; i++) {
        if (h->fan[i]) cudaStreamDestroy(h->fan[i]);
        if (h->fan_ev[i]) cudaEventDestroy(h->fan_ev[i]);
        h->fan[i] = nullptr;
        h->fan_ev[i] = nullptr;
    }
}

// ---- basis validation and pair construction ------------------------------------
static int validate_basis(const BasisHost &b) {
    if (b.nsh <= 0 || b.natoms <= 0 || b.num_bas <= 0 || b.mxgtot <= 0)
        return fail(LIBERI_E_ARG, "liberi_setup: non-positive size (nsh=%d natoms=%d num_bas=%d mxgtot=%d)",
                    b.nsh, b.natoms, b.num_bas, b.mxgtot);
    const long long ncoef = (long long)b.nsh * b.mxgtot;
    for (int s = 0; s < b.nsh; s++) {
        int l = b.ang_mom[s];
        if (l < 1 || l > 4) return fail(LIBERI_E_ARG, "liberi_setup: ang_mom(%d)=%d out of range", s + 1, l);
        if (l == 4 && b.cf.size() < (size_t)ncoef)
            return fail(LIBERI_E_ARG, "liberi_setup: shell %d is an f shell but contr_coef_f is null", s + 1);
        if (b.contr_num[s] < 1 || b.contr_num[s] > b.mxgtot)
            return fail(LIBERI_E_ARG, "liberi_setup: contr_num(%d)=%d out of range", s + 1, b.contr_num[s]);
        if (b.sh_loc[s] < 1 || b.sh_loc[s] - 1 + b.contr_num[s] > ncoef)
            return fail(LIBERI_E_ARG, "liberi_setup: sh_loc(%d)=%d out of range", s + 1, b.sh_loc[s]);
        if (b.atom_num[s] < 1 || b.atom_num[s] > b.natoms)
            return fail(LIBERI_E_ARG, "liberi_setup: atom_num(%d)=%d out of range", s + 1, b.atom_num[s]);
        int nc = l * (l + 1) / 2;
        if (b.atom_loc[s] < 1 || b.atom_loc[s] - 1 + nc > b.num_bas)
            return fail(LIBERI_E_ARG, "liberi_setup: atom_loc(%d)=%d out of range", s + 1, b.atom_loc[s]);
    }
    for (double x : b.schwrz)
        if (!(x >= 0.0)) return fail(LIBERI_E_ARG, "liberi_setup: negative or NaN Schwarz value");
    // the packed length n(n+1)/2 must fit the int32 matrix_size of
    // liberi_fock_build; device packed indices are unsigned 32-bit
    if (b.num_bas > 65535)
        return fail(LIBERI_E_UNSUPPORTED, "liberi_setup: num_bas %d exceeds 65535", b.num_bas);
    return LIBERI_OK;
}

static void build_pairs(const BasisHost &b, PairsHost &pr, std::vector<double4> &shell_xyz) {
    shell_xyz.resize(b.nsh);
    for (int s = 0; s < b.nsh; s++) {
        int a = b.atom_num[s] - 1;
        shell_xyz[s] = make_double4(b.coords[3 * a], b.coords[3 * a + 1], b.coords[3 * a + 2], 0.0);
    }
    // ascending per-L lists (classify_shells, liberi_shell_pair.F90:301-344)
    std::vector<int> lst[MAXL + 1];
    for (int s = 0; s < b.nsh; s++) lst[b.ang_mom[s] - 1].push_back(s);
    const std::vector<double> *coef[MAXL + 1] = {&b.cs, &b.cp, &b.cd, &b.cf};
    pr = PairsHost{};
    for (int l = 0; l <= MAXL; l++) pr.nl[l] = (int)lst[l].size();
    for (int c = 0; c < NPC; c++) {
        pr.class_off[c] = (int)pr.ish.size();
        const int l1 = PC_L1[c], l2 = PC_L2[c];
        const bool same = (l1 == l2);
        for (size_t ii = 0; ii < lst[l1].size(); ii++) {
            size_t jmax = same ? ii + 1 : lst[l2].size();
            for (size_t jj = 0; jj < jmax; jj++) {
                int is = lst[l1][ii], js = lst[l2][jj];
                int hi = std::max(is, js) + 1, lo = std::min(is, js) + 1;
                pr.ish.push_back(is);
                pr.jsh.push_back(js);
                pr.xint.push_back(b.schwrz[(size_t)hi * (hi - 1) / 2 + lo - 1]);
                // engine orientation: higher L first (same L: reference order)
                int A = is, B = js;
                if (l2 > l1) std::swap(A, B);
                pr.shell.push_back(make_int2(A, B));
                pr.prim0.push_back((int)pr.X.size());
                pr.kab.push_back(b.contr_num[is] * b.contr_num[js]);
                double r2 = 0.0;
                for (int x = 0; x < 3; x++) {
                    double d = b.coords[3 * (b.atom_num[js] - 1) + x] - b.coords[3 * (b.atom_num[is] - 1) + x];
                    r2 += d * d;
                }
                const double4 RA = shell_xyz[is], RB = shell_xyz[js];
                int kept = 0;
                for (int i = 0; i < b.contr_num[is]; i++) {
                    double a = b.exponents[b.sh_loc[is] - 1 + i];
                    double ca = (*coef[l1])[b.sh_loc[is] - 1 + i];
                    for (int j = 0; j < b.contr_num[js]; j++) {
                        double bb = b.exponents[b.sh_loc[js] - 1 + j];
                        double cb = (*coef[l2])[b.sh_loc[js] - 1 + j];
                        double p = a + bb, ip = 1.0 / p;
                        double mur2 = r2 * (a * ip) * bb;
                        // mu R^2 > cux pairs are skipped by the reference's
                        // rotated-axis kernels (int0000.F90:208-210) and
                        // contribute < e^-50 in its Rys kernels
                        if (mur2 > CUX) continue;
                        pr.P.push_back(make_double4((a * RA.x + bb * RB.x) * ip, (a * RA.y + bb * RB.y) * ip,
                                                    (a * RA.z + bb * RB.z) * ip, p));
                        pr.X.push_back(make_double2(SQRT_TWOPI52 * ca * cb * std::exp(-mur2) * ip, 0.5 * ip));
                        kept++;
                    }
                }
                pr.nprim.push_back(kept);
            }
        }
    }
    pr.class_off[NPC] = (int)pr.ish.size();
}

// ---- per-kernel plan ----------------------------------------------------------
static double class_max(const PairsHost &pr, int c) {
    double m = -HUGE_VAL;
    for (int i = pr.class_off[c]; i < pr.class_off[c + 1]; i++) m = std::max(m, pr.xint[i]);
    return m;
}

// static CTA tasks of a plan: chunks of at most ph.chunk kets per item; the
// capacity of the mixed tier's per-build lists follows
static void build_tasks(PlanHost &ph) {
    ph.tasks.clear();
    ph.task_cap = 0;
    for (const int4 &it : ph.items) {
        for (int k0 = 0; k0 < it.z; k0 += ph.chunk)
            ph.tasks.push_back(make_int4(it.x, it.y + k0, std::min(ph.chunk, it.z - k0), 0));
        ph.task_cap += (it.z + ph.chunk - 1) / ph.chunk + 1;
    }
}

static void build_plan(const PairsHost &pr, int k, double cut, int chunk, PlanHost &ph) {
    const KernelDesc &kd = KDESC[k];
    ph = PlanHost();
    ph.chunk = chunk;
    const int nb_all = pr.class_off[kd.bra + 1] - pr.class_off[kd.bra];
    const int nk_all = pr.class_off[kd.ket + 1] - pr.class_off[kd.ket];
    if (nb_all == 0 || nk_all == 0) return;
    const double sb = cut / class_max(pr, kd.cross ? kd.ket : kd.bra);
    const double sk = cut / class_max(pr, kd.cross ? kd.bra : kd.ket);
    std::vector<int> lb, lk;  // compacted lists, reference order (global ids)
    for (int i = pr.class_off[kd.bra]; i < pr.class_off[kd.bra + 1]; i++)
        if (pr.xint[i] >= sb) lb.push_back(i);
    if (kd.tri) lk = lb;
    else
        for (int i = pr.class_off[kd.ket]; i < pr.class_off[kd.ket + 1]; i++)
            if (pr.xint[i] >= sk) lk.push_back(i);
    if (lb.empty() || lk.empty()) return;
    ph.nbra_ref = (int)lb.size();
    ph.nket_ref = (int)lk.size();
    ph.ntot_ref = kd.tri ? (long long)lb.size() : (long long)lb.size() * (long long)lk.size();
    // engine rows: the reference's ket list for swapped classes (the
    // surviving partners of any element still form a prefix of the other
    // Schwarz-sorted list, and the quartet set is symmetric)
    if (kd.swap) std::swap(lb, lk);
    auto sorted = [&](const std::vector<int> &l, std::vector<int> &ids, std::vector<int> &orig,
                      std::vector<double> &x) {
        std::vector<int> ord(l.size());
        std::iota(ord.begin(), ord.end(), 0);
        // contraction-pattern groups (uniform primitive loops per CTA), each
        // sorted by Schwarz value: the partners of any pair are a prefix of
        // every group
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
            if (pr.kab[l[a]] != pr.kab[l[b]]) return pr.kab[l[a]] > pr.kab[l[b]];
            return pr.xint[l[a]] > pr.xint[l[b]];
        });
        for (int o : ord) {
            ids.push_back(l[o]);
            orig.push_back(o);
            x.push_back(pr.xint[l[o]]);
        }
    };
    sorted(lb, ph.bra_ids, ph.bra_orig, ph.bra_x);
    sorted(lk, ph.ket_ids, ph.ket_orig, ph.ket_x);
    ph.nbra = (int)ph.bra_ids.size();
    ph.nket = (int)ph.ket_ids.size();
    ph.ncount.assign(ph.nbra, 0);
    ph.pref.assign(ph.nbra + 1, 0);
    // ket segments of equal contraction pattern
    std::vector<int> seg{0};
    for (int j = 1; j < ph.nket; j++)
        if (pr.kab[ph.ket_ids[j]] != pr.kab[ph.ket_ids[j - 1]]) seg.push_back(j);
    seg.push_back(ph.nket);
    ph.items.clear();
    for (int i = 0; i < ph.nbra; i++) {
        const double xb = ph.bra_x[i];
        int n_i = 0;
        for (size_t g = 0; g + 1 < seg.size(); g++) {
            const int s = seg[g], e = seg[g + 1];
            if (kd.tri && s > i) break;  // triangle: partners at positions <= i
            int lo = s, hi = e;
            while (lo < hi) {
                int mid = (lo + hi) / 2;
                double t = xb * ph.ket_x[mid];
                bool pass = kd.op == OP_GE ? (t >= cut) : (kd.op == OP_GT ? (t > cut) : true);
                if (pass) lo = mid + 1; else hi = mid;
            }
            int n = lo - s;
            if (kd.tri) n = std::min(n, i - s + 1);
            if (n > 0) {
                ph.items.push_back(make_int4(i, s, n, 0));
                n_i += n;
            }
        }
        ph.ncount[i] = n_i;
        ph.pref[i + 1] = ph.pref[i] + n_i;
    }
    ph.total = ph.pref[ph.nbra];
    if (ph.chunk <= 0) ph.chunk = default_chunk(k);
    build_tasks(ph);
}

// Cost-balanced rank split: this rank keeps the contiguous run of items
// whose cost midpoints fall in its 1/nsize share of the class's primitive-
// quartet total (cost of an item: nprim(row pair) x sum of its kets' nprim).
static void balance_items(const PairsHost &pr, int rank, int nsize, PlanHost &ph) {
    std::vector<double> cost(ph.items.size());
    double total = 0.0;
    for (size_t i = 0; i < ph.items.size(); i++) {
        const int4 &it = ph.items[i];
        double kc = 0.0;
        for (int j = it.y; j < it.y + it.z; j++) kc += pr.nprim[ph.ket_ids[j]];
        cost[i] = (double)pr.nprim[ph.bra_ids[it.x]] * kc + 1.0;  // + 1: empty-primitive pairs still cost
        total += cost[i];
    }
    std::vector<int4> mine;
    double before = 0.0;
    for (size_t i = 0; i < ph.items.size(); i++) {
        const double mid = (before + 0.5 * cost[i]) / total * nsize;
        if ((int)mid == rank || (rank == nsize - 1 && mid >= nsize)) mine.push_back(ph.items[i]);
        before += cost[i];
    }
    ph.items.swap(mine);
    build_tasks(ph);
}

// Every class's plan (and, for the balanced rank split, this rank's slice of
// it) on up to one host thread per class: each reads the pairs and writes
// only its own plan.  C60's 21 plans took 42 ms on one thread.
static void build_plans(const PairsHost &pr, double cut, const int *chunk, int rank_split, int rank, int nprocs,
                        PlanHost *plans) {
    auto one = [&](int k) {
        const bool run = (k == 0 && pr.nl[0] > 0) || (k >= 1 && k <= 5 && pr.nl[1] > 0) ||
                         (k >= 6 && k < NKERN && pr.nl[2] > 0) || (k >= NKERN && pr.nl[3] > 0);
        if (!run) {
            plans[k] = PlanHost();
            return;
        }
        build_plan(pr, k, cut, chunk ? chunk[k] : 0, plans[k]);
        if (rank_split == 1 && nprocs > 1) balance_items(pr, rank, nprocs, plans[k]);
    };
    std::atomic<int> next{0};
    auto worker = [&]() {
        for (int k = next++; k < NKALL; k = next++) one(k);
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const int nextra = (int)std::min<unsigned>(pr.nl[3] > 0 ? NKALL : NKERN, hw > 1 ? hw : 1) - 1;
    std::vector<std::thread> pool;
    for (int t = 0; t < nextra; t++) {
        try {
            pool.emplace_back(worker);
        } catch (const std::system_error &) {
            break;  // no more host threads: the calling thread does the rest
        }
    }
    worker();
    for (std::thread &th : pool) th.join();
}

static void make_tasks(const PlanHost &ph, int chunk, int mol, std::vector<int4> &out) {
    for (const int4 &it : ph.items)
        for (int k0 = 0; k0 < it.z; k0 += chunk) out.push_back(make_int4(it.x, it.y + k0, std::min(chunk, it.z - k0), mol));
}

// Ket records of a plan (layout beside KET_REC): C - D, C, the first basis
// functions of C and D and the ket pair's primitive range, per ket position.
static void build_ket_records(const BasisHost &b, const PairsHost &pr, const std::vector<int> &ket_ids,
                              std::vector<double4> &rec) {
    auto bits = [](unsigned lo, unsigned hi) {
        const unsigned long long v = (unsigned long long)lo | ((unsigned long long)hi << 32);
        double d;
        std::memcpy(&d, &v, sizeof d);
        return d;
    };
    rec.resize(KET_REC * ket_ids.size());
    for (size_t j = 0; j < ket_ids.size(); j++) {
        const int Q = ket_ids[j];
        const int C = pr.shell[Q].x, D = pr.shell[Q].y;
        const double *xc = &b.coords[3 * (size_t)(b.atom_num[C] - 1)];
        const double *xd = &b.coords[3 * (size_t)(b.atom_num[D] - 1)];
        rec[KET_REC * j] = make_double4(xc[0] - xd[0], xc[1] - xd[1], xc[2] - xd[2], xc[0]);
        rec[KET_REC * j + 1] = make_double4(xc[1], xc[2], bits(b.atom_loc[C] - 1, b.atom_loc[D] - 1),
                                            bits(pr.prim0[Q], pr.nprim[Q]));
    }
}

static size_t plan_device_bytes(const PlanHost &ph);

static int upload_plans(liberi_handle h) {
    size_t total = 0;
    for (int k = 0; k < NKALL; k++) total += plan_device_bytes(h->plan[k]);
    CUDA_TRY(arena_open(h, h->arena_plans, total));
    ArenaScope scope{h};
    for (int k = 0; k < NKALL; k++) {
        PlanHost &ph = h->plan[k];
        if (ph.nbra == 0) continue;
        {
            std::vector<double4> rec;
            build_ket_records(h->basis, h->pairs, ph.ket_ids, rec);
            CUDA_TRY(dev_upload(h, &ph.d_ket_rec, rec.data(), rec.size()));
        }
        CUDA_TRY(dev_upload(h, &ph.d_bra, ph.bra_ids.data(), ph.bra_ids.size()));
        CUDA_TRY(dev_upload(h, &ph.d_ket, ph.ket_ids.data(), ph.ket_ids.size()));
        CUDA_TRY(dev_upload(h, &ph.d_bra_orig, ph.bra_orig.data(), ph.bra_orig.size()));
        CUDA_TRY(dev_upload(h, &ph.d_ket_orig, ph.ket_orig.data(), ph.ket_orig.size()));
        CUDA_TRY(dev_upload(h, &ph.d_bra_x, ph.bra_x.data(), ph.bra_x.size()));
        CUDA_TRY(dev_upload(h, &ph.d_ket_x, ph.ket_x.data(), ph.ket_x.size()));
        CUDA_TRY(dev_upload(h, &ph.d_items, ph.items.data(), ph.items.size()));
        CUDA_TRY(dev_upload(h, &ph.d_tasks, ph.tasks.data(), ph.tasks.size()));
        CUDA_TRY(dev_alloc(h, &ph.d_tasks64, (size_t)ph.task_cap));
        CUDA_TRY(dev_alloc(h, &ph.d_tasks32, (size_t)ph.task_cap));
        CUDA_TRY(dev_alloc(h, &ph.d_ntasks, 4));
    }
    return LIBERI_OK;
}

// Device bytes that upload_plans allocates for one class plan.
static size_t plan_device_bytes(const PlanHost &ph) {
    if (ph.nbra == 0) return 0;
    return up_bytes(KET_REC * ph.ket_ids.size(), sizeof(double4)) + up_bytes(ph.bra_ids.size(), sizeof(int)) +
           up_bytes(ph.ket_ids.size(), sizeof(int)) + up_bytes(ph.bra_orig.size(), sizeof(int)) +
           up_bytes(ph.ket_orig.size(), sizeof(int)) + up_bytes(ph.bra_x.size(), sizeof(double)) +
           up_bytes(ph.ket_x.size(), sizeof(double)) + up_bytes(ph.items.size(), sizeof(int4)) +
           up_bytes(ph.tasks.size(), sizeof(int4)) + 2 * al_bytes((size_t)ph.task_cap, sizeof(int4)) +
           al_bytes(4, sizeof(int));
}

// Device bytes that upload_basis allocates.
static size_t basis_device_bytes(const BasisHost &b, const PairsHost &pr) {
    const size_t npair = pr.shell.size(), nprim = pr.P.size(), nsh = (size_t)b.nsh;
    const size_t ntri = (size_t)b.num_bas * (b.num_bas + 1) / 2, nsq = (size_t)b.num_bas * b.num_bas;
    return up_bytes(nsh, sizeof(double4)) + up_bytes(nsh, sizeof(int)) + up_bytes(npair, sizeof(int2)) +
           2 * up_bytes(npair, sizeof(int)) + up_bytes(nprim, sizeof(double4)) + up_bytes(nprim, sizeof(double2)) +
           up_bytes(2 * nprim, sizeof(float4)) + up_bytes(RYS_TABLE_SIZE, sizeof(double)) +
           up_bytes(RYSF_TABLE_SIZE, sizeof(float)) + 2 * al_bytes(ntri, sizeof(double)) +
           al_bytes(nsq, sizeof(double)) + al_bytes(nsq, sizeof(float)) + al_bytes(1, sizeof(unsigned long long)) +
           al_bytes(nprim, sizeof(float)) + (pr.nl[3] > 0 ? up_bytes(RYS7_TABLE_SIZE, sizeof(double)) : 0);
}

static void compute_stats(liberi_handle h) {
    for (int k = 0; k < NKALL; k++) {
        const PlanHost &ph = h->plan[k];
        long long q = 0;
        for (const int4 &it : ph.items) q += it.z;
        if (k >= NKERN) h->fq[k - NKERN] = q;
        else h->stats.quartets[k] = q;  // this rank's share under the balanced split
        // primitive quartets: sum_i nprim(bra_i) * sum_{j<n_i} nprim(ket_j)
        std::vector<long long> kp(ph.nket + 1, 0);
        for (int j = 0; j < ph.nket; j++) kp[j + 1] = kp[j] + h->pairs.nprim[ph.ket_ids[j]];
        long long s = 0;
        for (const int4 &it : ph.items)
            s += (long long)h->pairs.nprim[ph.bra_ids[it.x]] * (kp[it.y + it.z] - kp[it.y]);
        if (k >= NKERN) h->fprim[k - NKERN] = s;
        else h->stats.prim_quartets[k] = s;
    }
}

static int copy_basis(BasisHost &b, int nsh, int natoms, int num_bas, int mxgtot, const int32_t *ang_mom,
                      const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                      const int32_t *atom_loc, const int32_t *start_bas, const int32_t *end_bas,
                      const double *exponents, const double *cs, const double *cp, const double *cd,
                      const double *cf, const double *coords, const double *schwrz) {
    if (nsh <= 0 || natoms <= 0 || num_bas <= 0 || mxgtot <= 0)
        return fail(LIBERI_E_ARG, "liberi_setup: non-positive size (nsh=%d natoms=%d num_bas=%d mxgtot=%d)",
                    nsh, natoms, num_bas, mxgtot);
    if (!ang_mom || !contr_num || !sh_loc || !atom_num || !atom_loc || !exponents || !cs || !cp || !cd ||
        !coords || !schwrz)
        return fail(LIBERI_E_ARG, "liberi_setup: null array argument");
    const size_t ncoef = (size_t)nsh * mxgtot;
    b.nsh = nsh;
    b.natoms = natoms;
    b.num_bas = num_bas;
    b.mxgtot = mxgtot;
    b.ang_mom.assign(ang_mom, ang_mom + nsh);
    b.contr_num.assign(contr_num, contr_num + nsh);
    b.sh_loc.assign(sh_loc, sh_loc + nsh);
    b.atom_num.assign(atom_num, atom_num + nsh);
    b.atom_loc.assign(atom_loc, atom_loc + nsh);
    if (start_bas) b.start_bas.assign(start_bas, start_bas + nsh);
    if (end_bas) b.end_bas.assign(end_bas, end_bas + nsh);
    b.exponents.assign(exponents, exponents + ncoef);
    b.cs.assign(cs, cs + ncoef);
    b.cp.assign(cp, cp + ncoef);
    b.cd.assign(cd, cd + ncoef);
    if (cf) b.cf.assign(cf, cf + ncoef);
    b.coords.assign(coords, coords + 3 * (size_t)natoms);
    b.schwrz.assign(schwrz, schwrz + (size_t)nsh * (nsh + 1) / 2);
    return LIBERI_OK;
}

static size_t basis_device_bytes(const BasisHost &b, const PairsHost &pr);

static DevBasis dev_basis(liberi_handle h);

static int upload_basis(liberi_handle h, const std::vector<double4> &shell_xyz) {
    const BasisHost &b = h->basis;
    CUDA_TRY(arena_open(h, h->arena_basis, basis_device_bytes(b, h->pairs)));
    ArenaScope scope{h};
    std::vector<int> bf0(b.nsh);
    for (int s = 0; s < b.nsh; s++) bf0[s] = b.atom_loc[s] - 1;
    CUDA_TRY(dev_upload(h, &h->dev.shell_xyz, shell_xyz.data(), shell_xyz.size()));
    CUDA_TRY(dev_upload(h, &h->dev.shell_bf0, bf0.data(), bf0.size()));
    CUDA_TRY(dev_upload(h, &h->dev.pair_shell, h->pairs.shell.data(), h->pairs.shell.size()));
    CUDA_TRY(dev_upload(h, &h->dev.pair_prim0, h->pairs.prim0.data(), h->pairs.prim0.size()));
    CUDA_TRY(dev_upload(h, &h->dev.pair_nprim, h->pairs.nprim.data(), h->pairs.nprim.size()));
    CUDA_TRY(dev_upload(h, &h->dev.prim_P, h->pairs.P.data(), h->pairs.P.size()));
    CUDA_TRY(dev_upload(h, &h->dev.prim_X, h->pairs.X.data(), h->pairs.X.size()));
    const std::vector<double> &tab = rys_table_host();
    CUDA_TRY(dev_upload(h, &h->d_tab, tab.data(), tab.size()));
    const std::vector<float> &tabf = rys_table_f32_host();
    CUDA_TRY(dev_upload(h, &h->d_tabf, tabf.data(), tabf.size()));
    if (h->pairs.nl[3] > 0) {
        const std::vector<double> &tab7 = rys_table7_host();
        CUDA_TRY(dev_upload(h, &h->d_tab7, tab7.data(), tab7.size()));
    }
    // Bounds of the single primitive pairs (the FP32 tier's primitive
    // screening), computed on the device from the pair data and tables; then
    // every pair's primitives are put in order of decreasing bound, so that
    // the FP32 loops stop at the first primitive below the cut.  The FP64
    // sums only change order.
    PairsHost &pr = h->pairs;
    const size_t nprim = pr.P.size();
    CUDA_TRY(dev_alloc(h, &h->dev.prim_bound, nprim));
    std::vector<float> bound(nprim);
    if (nprim) {
        DevBasis db = dev_basis(h);
        for (int c = 0; c < NPC_SPD; c++) {
            const int o = pr.class_off[c], n = pr.class_off[c + 1] - o;
            CUDA_TRY(launch_prim_bound(c, n, o, db, h->d_tab, h->dev.prim_bound, h->stream));
        }
        CUDA_TRY(cudaMemcpyAsync(bound.data(), h->dev.prim_bound, nprim * sizeof(float), cudaMemcpyDeviceToHost,
                                 h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        // f pairs (FP64 only) have no bounds: their primitives keep their order
        for (int q = pr.class_off[NPC_SPD]; q < pr.class_off[NPC]; q++)
            for (int k = pr.prim0[q]; k < pr.prim0[q] + pr.nprim[q]; k++) bound[k] = 0.0f;
        std::vector<int> ord;
        std::vector<double4> P2(pr.P.size());
        std::vector<double2> X2(pr.X.size());
        std::vector<float> bound2(nprim);
        for (size_t q = 0; q < pr.shell.size(); q++) {
            const int k0 = pr.prim0[q], n = pr.nprim[q];
            ord.resize(n);
            std::iota(ord.begin(), ord.end(), k0);
            std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return bound[x] > bound[y]; });
            for (int i = 0; i < n; i++) {
                P2[k0 + i] = pr.P[ord[i]];
                X2[k0 + i] = pr.X[ord[i]];
                bound2[k0 + i] = bound[ord[i]];
            }
        }
        pr.P.swap(P2);
        pr.X.swap(X2);
        bound.swap(bound2);
        CUDA_TRY(cudaMemcpyAsync(h->dev.prim_P, pr.P.data(), nprim * sizeof(double4), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(cudaMemcpyAsync(h->dev.prim_X, pr.X.data(), nprim * sizeof(double2), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(cudaMemcpyAsync(h->dev.prim_bound, bound.data(), nprim * sizeof(float), cudaMemcpyHostToDevice,
                                 h->stream));
    }
    {  // FP32 tier copies: P - A is formed in FP64 and rounded once
        std::vector<float4> paf(2 * pr.P.size());
        for (size_t q = 0; q < pr.shell.size(); q++) {
            const double4 A = shell_xyz[pr.shell[q].x];
            for (int k = pr.prim0[q]; k < pr.prim0[q] + pr.nprim[q]; k++) {
                const double4 P = pr.P[k];
                paf[2 * k] = make_float4((float)P.x, (float)P.y, (float)P.z, (float)P.w);
                paf[2 * k + 1] = make_float4((float)(P.x - A.x), (float)(P.y - A.y), (float)(P.z - A.z), (float)pr.X[k].x);
            }
        }
        CUDA_TRY(dev_upload(h, &h->dev.prim_PAf, paf.data(), paf.size()));
    }
    const size_t ntri = (size_t)b.num_bas * (b.num_bas + 1) / 2;
    CUDA_TRY(dev_alloc(h, &h->dev.D, ntri));
    CUDA_TRY(dev_alloc(h, &h->dev.F, ntri));
    const size_t nsq = (size_t)b.num_bas * b.num_bas;
    CUDA_TRY(dev_alloc(h, &h->dev.Dsq, nsq));
    CUDA_TRY(dev_alloc(h, &h->dev.Df, nsq));
    CUDA_TRY(dev_alloc(h, &h->d_maxd, 1));
    // the host copies above are pageable: the uploads complete before return
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return LIBERI_OK;
}

static DevBasis dev_basis(liberi_handle h) {
    DevBasis d;
    d.shell_xyz = h->dev.shell_xyz;
    d.shell_bf0 = h->dev.shell_bf0;
    d.pair_shell = h->dev.pair_shell;
    d.pair_prim0 = h->dev.pair_prim0;
    d.pair_nprim = h->dev.pair_nprim;
    d.prim_P = h->dev.prim_P;
    d.prim_X = h->dev.prim_X;
    d.prim_PAf = h->dev.prim_PAf;
    d.prim_bound = h->dev.prim_bound;
    return d;
}

// ---- build ------------------------------------------------------------------------
static int replan(liberi_handle h) {
    bool had_plans = false;
    for (int k = 0; k < NKALL; k++) had_plans = had_plans || h->plan[k].d_bra != nullptr;
    // builds of the old plans may still run on any stream (re-plans follow an
    // option change, rarely): wait for the device before releasing them
    if (had_plans) CUDA_TRY(cudaDeviceSynchronize());
    for (int k = 0; k < NKALL; k++) {
        PlanHost &ph = h->plan[k];
        // pieces of the plan arena are released with it; a task list the
        // tuner uploaded on its own is released here
        for (void *p : {(void *)ph.d_ket_rec, (void *)ph.d_bra, (void *)ph.d_ket, (void *)ph.d_bra_orig,
                        (void *)ph.d_ket_orig, (void *)ph.d_bra_x, (void *)ph.d_ket_x, (void *)ph.d_items,
                        (void *)ph.d_tasks, (void *)ph.d_tasks64, (void *)ph.d_tasks32, (void *)ph.d_ntasks})
            if (p) dev_release(h, p);
    }
    if (h->arena_plans.base) dev_release(h, h->arena_plans.base);
    h->arena_plans = liberi_handle_s::Arena();
    h->dev.bytes = h->arena_basis.size;
    build_plans(h->pairs, h->schwarz_cut, h->chunk, h->rank_split, h->my_rank, h->num_procs, h->plan);
    int rc = upload_plans(h);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));  // plans visible to builds on other streams
    compute_stats(h);
    h->stats.device_bytes = (int64_t)h->dev.bytes;
    h->plan_dirty = false;
    return LIBERI_OK;
}

// The reference's rank split of class k as the class kernels apply it
// (balanced split: the plan already holds only this rank's items).
static RankSplit rank_split_of(liberi_handle h, int k) {
    const KernelDesc &kd = KDESC[k];
    const PlanHost &ph = h->plan[k];
    RankSplit rs;
    rs.rank = h->my_rank;
    rs.nsize = h->rank_split == 1 ? 1 : h->num_procs;
    rs.tile = kd.tile;
    rs.ntot = ph.ntot_ref;
    rs.nbra_ref = ph.nbra_ref;
    rs.nket_ref = ph.nket_ref;
    rs.tri = kd.tri;
    rs.ketmajor = kd.ketmajor;
    return rs;
}

// Device lists of class k's plan (the task list is filled in by the caller).
static DevPlan dev_plan_of(liberi_handle h, int k) {
    const PlanHost &ph = h->plan[k];
    DevPlan dp;
    dp.bra_ids = ph.d_bra;
    dp.ket_ids = ph.d_ket;
    dp.ket_rec = ph.d_ket_rec;
    dp.bra_orig = ph.d_bra_orig;
    dp.ket_orig = ph.d_ket_orig;
    dp.tasks = ph.d_tasks;
    dp.ntasks_dev = nullptr;
    dp.ntasks = (int)ph.tasks.size();
    dp.swapped = KDESC[k].swap;
    return dp;
}

// One Fock build on device buffers.  Closed shell (dDb null): F = J(D) - K(D)
// in the reference's DIRFCK units.  Open shell (dDb non-null, spin 0 or 1):
// F_spin = J(D + Db) - K(2 D_spin), D the alpha density: the kernels read the
// Coulomb density and, k_offset further on, the exchange density.
static int build_on_device(liberi_handle h, const double *dD, double *dF, cudaStream_t st,
                           const double *dDb = nullptr, int spin = 0) {
    if (h->plan_dirty) {
        int rc = replan(h);
        if (rc) return rc;
    }
    h->last_split_lists = h->precision == 1;
    const BasisHost &b = h->basis;
    const long long ntri = (long long)b.num_bas * (b.num_bas + 1) / 2;
    CUDA_TRY(cudaMemsetAsync(dF, 0, ntri * sizeof(double), st));  // liberi_driver.F90:64
    LaunchCtx ctx;
    ctx.basis = dev_basis(h);
    ctx.rys_tab = h->d_tab;
    ctx.rys_tabf = h->d_tabf;
    ctx.D = h->dev.Dsq;
    ctx.F = dF;
    ctx.schwarz_cut = h->schwarz_cut;
    ctx.eri_cut = h->eri_cut;
    ctx.stream = st;
    ctx.num_sms = h->num_sms;
    const bool mixed = h->precision == 1;
    ctx.Df = h->dev.Df;
    ctx.maxd = mixed ? h->d_maxd : nullptr;
    ctx.prim_cut = mixed ? h->fp32_prim * h->fp32_cut : 0.0;
    if (!dDb) {
        // the class kernels read D as a full matrix (and in float for the FP32 tier)
        CUDA_TRY(launch_unpack(dD, b.num_bas, h->dev.Dsq, mixed ? h->dev.Df : nullptr, st));
        if (mixed) CUDA_TRY(launch_maxabs(dD, ntri, h->d_maxd, st));
    } else {
        const size_t nsq = (size_t)b.num_bas * b.num_bas;
        if (!h->dev.uhf_sq) {  // first open-shell build of this handle
            CUDA_TRY(cudaMallocAsync((void **)&h->dev.uhf_sq, 2 * nsq * sizeof(double), h->stream));
            h->allocs.push_back(h->dev.uhf_sq);
            CUDA_TRY(cudaMallocAsync((void **)&h->dev.uhf_sqf, 2 * nsq * sizeof(float), h->stream));
            h->allocs.push_back(h->dev.uhf_sqf);
            CUDA_TRY(cudaStreamSynchronize(h->stream));
        }
        CUDA_TRY(launch_unpack_combo(dD, dDb, 1.0, 1.0, b.num_bas, h->dev.uhf_sq, mixed ? h->dev.uhf_sqf : nullptr, st));
        CUDA_TRY(launch_unpack_combo(dD, dDb, spin == 0 ? 2.0 : 0.0, spin == 0 ? 0.0 : 2.0, b.num_bas,
                                     h->dev.uhf_sq + nsq, mixed ? h->dev.uhf_sqf + nsq : nullptr, st));
        // the mixed tier's bound uses the largest element of both densities
        if (mixed) CUDA_TRY(launch_maxabs(h->dev.uhf_sq, (long long)(2 * nsq), h->d_maxd, st));
        ctx.D = h->dev.uhf_sq;
        ctx.Df = h->dev.uhf_sqf;
        ctx.k_offset = nsq;
    }
    for (int k = 0; k < NKERN; k++) h->ev_recorded[k] = false;
    // mixed precision: every class's FP64 task list (the few quartets above
    // fp32_cut, the costliest ones, in small low-occupancy launches) runs on
    // the side stream beside the FP32 lists on the build's stream.  Measured
    // on C60: 1.5 ms faster at cut 1e-2 than running them in turn, where
    // putting the high-L classes on the side instead gained 1 ms; FP64
    // builds put the classes of side_mask there (the small low-occupancy
    // classes and the seven Rys classes, measured against the kernel shapes
    // of this build).  The task splits of every class come first; per-class
    // timing keeps one stream.
    // Small builds (few quartets) are a sequence of class kernels each as long
    // as its costliest quartet's primitive loop: their classes are spread over
    // FAN_STREAMS streams instead (measured: 42 functions 2.9 -> 1.0 ms, 366
    // functions 5.1 -> 3.9 ms; C60, 2.6e8 quartets, 107 -> 121 ms, hence the
    // size limit).
    long long nquart = 0;
    for (int k = 0; k < NKERN; k++)
        if ((h->class_mask >> k) & 1u) nquart += h->stats.quartets[k];
    const bool fan = h->fan_out && h->overlap && !h->timing && nquart <= FAN_MAX_QUARTETS;
    const bool fork = h->overlap && !h->timing && !fan;
    const uint32_t side64 = mixed ? 0u : h->side_mask;
    if (fan) {
        if (mixed)
            for (int k = 0; k < NKERN; k++) {
                PlanHost &ph = h->plan[k];
                if (ph.total == 0 || !((h->class_mask >> k) & 1u)) continue;
                CUDA_TRY(launch_split_tasks((int)ph.items.size(), ph.d_items, ph.d_bra_x, ph.d_ket_x, h->d_maxd,
                                            h->fp32_cut, ph.chunk, ph.d_tasks64, ph.d_tasks32, ph.d_ntasks, st));
            }
        if (!h->fork_ev) CUDA_TRY(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(h->fork_ev, st));
        for (int i = 0; i < FAN_STREAMS; i++) {
            if (!h->fan[i]) {
                CUDA_TRY(cudaStreamCreateWithFlags(&h->fan[i], cudaStreamNonBlocking));
                CUDA_TRY(cudaEventCreateWithFlags(&h->fan_ev[i], cudaEventDisableTiming));
            }
            CUDA_TRY(cudaStreamWaitEvent(h->fan[i], h->fork_ev, 0));
        }
    }
    int nfanned = 0;
    if (fork && mixed) {
        for (int k = 0; k < NKERN; k++) {
            PlanHost &ph = h->plan[k];
            if (ph.total == 0 || !((h->class_mask >> k) & 1u)) continue;
            CUDA_TRY(launch_split_tasks((int)ph.items.size(), ph.d_items, ph.d_bra_x, ph.d_ket_x, h->d_maxd,
                                        h->fp32_cut, ph.chunk, ph.d_tasks64, ph.d_tasks32, ph.d_ntasks, st));
        }
    }
    if (fork) {
        // each object is created once per handle (the fan-out path may have
        // made the fork event already)
        if (!h->side) CUDA_TRY(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        if (!h->fork_ev) CUDA_TRY(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
        if (!h->join_ev) CUDA_TRY(cudaEventCreateWithFlags(&h->join_ev, cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(h->fork_ev, st));
        CUDA_TRY(cudaStreamWaitEvent(h->side, h->fork_ev, 0));
    }
    // high-L classes (few quartets per row pair, a latency tail) first
    static const int ORDER[NKERN] = {20, 19, 18, 14, 11, 13, 10, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 15, 16, 17};
    for (int oi = 0; oi < NKERN; oi++) {
        const int k = ORDER[oi];
        PlanHost &ph = h->plan[k];
        if (ph.total == 0 || !((h->class_mask >> k) & 1u)) continue;
        const KernelDesc &kd = KDESC[k];
        ctx.stream = st;
        if (h->timing) {
            if (!h->ev[k][0]) {
                CUDA_TRY(cudaEventCreate(&h->ev[k][0]));
                CUDA_TRY(cudaEventCreate(&h->ev[k][1]));
            }
            CUDA_TRY(cudaEventRecord(h->ev[k][0], st));
        }
        const RankSplit rs = rank_split_of(h, k);
        DevPlan dp = dev_plan_of(h, k);
        const int nbf = b.num_bas;
        const size_t tile_bytes = (size_t)(ncart_l(kd.la) + ncart_l(kd.lb)) * nbf * sizeof(double);
        const int tile_rows = (tile_bytes <= TILE_MAX_BYTES && ((h->tile_mask >> k) & 1u)) ? 1 : 0;
        if (fan) {  // every launch of the class on its fan stream (task splits came first)
            ctx.stream = h->fan[nfanned++ % FAN_STREAMS];
            if (!mixed) {
                dp.tasks = ph.d_tasks;
                dp.ntasks_dev = nullptr;
                dp.ntasks = (int)ph.tasks.size();
                CUDA_TRY(launch_class(k, ctx, dp, rs, 0, nbf, tile_rows, h->variant[0][k]));
            } else {
                dp.ntasks = ph.task_cap;
                dp.tasks = ph.d_tasks64;
                dp.ntasks_dev = ph.d_ntasks;
                CUDA_TRY(launch_class(k, ctx, dp, rs, 0, nbf, tile_rows, h->variant[0][k]));
                dp.tasks = ph.d_tasks32;
                dp.ntasks_dev = ph.d_ntasks + 1;
                CUDA_TRY(launch_class(k, ctx, dp, rs, 1, nbf, tile_rows, h->variant[1][k]));
            }
            ctx.stream = st;
        } else if (!mixed) {
            dp.tasks = ph.d_tasks;
            dp.ntasks_dev = nullptr;
            dp.ntasks = (int)ph.tasks.size();
            ctx.stream = (fork && ((side64 >> k) & 1u)) ? h->side : st;
            CUDA_TRY(launch_class(k, ctx, dp, rs, 0, nbf, tile_rows, h->variant[0][k]));
            ctx.stream = st;
        } else {
            if (!fork)  // (fan and fork builds split every class first)
                CUDA_TRY(launch_split_tasks((int)ph.items.size(), ph.d_items, ph.d_bra_x, ph.d_ket_x, h->d_maxd,
                                            h->fp32_cut, ph.chunk, ph.d_tasks64, ph.d_tasks32, ph.d_ntasks, st));
            dp.ntasks = ph.task_cap;
            dp.tasks = ph.d_tasks64;
            dp.ntasks_dev = ph.d_ntasks;
            ctx.stream = fork ? h->side : st;
            CUDA_TRY(launch_class(k, ctx, dp, rs, 0, nbf, tile_rows, h->variant[0][k]));
            dp.tasks = ph.d_tasks32;
            dp.ntasks_dev = ph.d_ntasks + 1;
            ctx.stream = st;
            CUDA_TRY(launch_class(k, ctx, dp, rs, 1, nbf, tile_rows, h->variant[1][k]));
        }
        if (h->timing) {
            CUDA_TRY(cudaEventRecord(h->ev[k][1], st));
            h->ev_recorded[k] = true;
        }
    }
    // f classes (FP64 in every precision mode), in the driver's order
    if (h->pairs.nl[3] > 0) {
        ctx.rys_tab7 = h->d_tab7;
        for (int k = NKERN; k < NKALL; k++) {
            PlanHost &ph = h->plan[k];
            if (ph.total == 0) continue;
            DevPlan dp = dev_plan_of(h, k);
            ctx.stream = fan ? h->fan[nfanned++ % FAN_STREAMS] : st;
            CUDA_TRY(launch_fclass(k, ctx, dp, rank_split_of(h, k), b.num_bas));
        }
        ctx.stream = st;
    }
    if (fan)  // join: the build completes on the caller's stream
        for (int i = 0; i < FAN_STREAMS; i++) {
            CUDA_TRY(cudaEventRecord(h->fan_ev[i], h->fan[i]));
            CUDA_TRY(cudaStreamWaitEvent(st, h->fan_ev[i], 0));
        }
    if (fork) {  // join: the build completes on the caller's stream
        CUDA_TRY(cudaEventRecord(h->join_ev, h->side));
        CUDA_TRY(cudaStreamWaitEvent(st, h->join_ev, 0));
    }
    return LIBERI_OK;
}

// Internal helpers for the allocation-free Schwarz entry point (noalloc.cu):
// the same input checks and host-side pair construction as liberi_c_schwarz.
namespace liberi {
int schwarz_host_inputs(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot, const int32_t *ang_mom,
                        const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                        const int32_t *atom_loc, const double *exponents, const double *contr_coef_s,
                        const double *contr_coef_p, const double *contr_coef_d, const double *coords,
                        BasisHost &basis, PairsHost &pairs, std::vector<double4> &shell_xyz) {
    if (ang_mom)
        for (int s = 0; s < nsh; s++)
            if (ang_mom[s] == 4)
                return fail(LIBERI_E_UNSUPPORTED, "liberi_schwarz: shell %d is an f shell; the generator covers s/p/d", s + 1);
    std::vector<double> ones((size_t)(nsh > 0 ? nsh : 0) * (nsh + 1) / 2, 1.0);
    int rc = copy_basis(basis, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc,
                        nullptr, nullptr, exponents, contr_coef_s, contr_coef_p, contr_coef_d, nullptr, coords,
                        ones.data());
    if (rc) return rc;
    rc = validate_basis(basis);
    if (rc) return rc;
    build_pairs(basis, pairs, shell_xyz);
    return LIBERI_OK;
}

int set_error(int code, const char *msg) { return fail(code, "%s", msg); }
}  // namespace liberi


// ---- batched builds over several molecules ---------------------------------------
// One launch per class covers every molecule of the batch (the task's w field
// selects the molecule); one F-zeroing launch precedes them.  The sequence can
// be captured once into a CUDA graph and replayed every SCF iteration.
struct liberi_batch_s {
    std::vector<liberi_handle> hs;
    int device = 0;
    int nbf_max = 0;
    long long ntri_max = 0;
    MolView *d_mols = nullptr;
    ClassView *d_cv[NKERN] = {};
    int4 *d_tasks[NKERN] = {};
    int ntasks[NKERN] = {};
    int chunk[NKERN] = {};
    // mixed precision: every molecule's items per class (w = molecule), per-build task lists
    int precision = 0;
    double fp32_cut = 0.0, fp32_prim = 0.0;
    int4 *d_items[NKERN] = {};
    int nitems[NKERN] = {};
    int cap[NKERN] = {};
    int4 *d_t64[NKERN] = {}, *d_t32[NKERN] = {};
    int *d_counts[NKERN] = {};
    unsigned long long *d_maxd = nullptr;
    double *d_Dsq = nullptr;      // every molecule's D as a full matrix (offsets sq_off)
    float *d_Df = nullptr;        // mixed: the same in float
    std::vector<size_t> sq_off;
    bool bound = false;
    cudaStream_t stream = nullptr;
    // mixed: the FP64 lists run on a second stream beside the FP32 lists
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<void *> allocs;
};

static void batch_free(liberi_batch b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    for (void *p : b->allocs) cudaFree(p);
    b->allocs.clear();
    if (b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
    if (b->side) cudaStreamDestroy(b->side);
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    if (b->join_ev) cudaEventDestroy(b->join_ev);
    b->side = nullptr;
    b->fork_ev = b->join_ev = nullptr;
}

static int batch_build_tasks(liberi_batch b, int k) {
    std::vector<int4> tasks;
    for (size_t m = 0; m < b->hs.size(); m++) make_tasks(b->hs[m]->plan[k], b->chunk[k], (int)m, tasks);
    if (b->d_tasks[k]) {
        cudaFree(b->d_tasks[k]);
        b->allocs.erase(std::remove(b->allocs.begin(), b->allocs.end(), (void *)b->d_tasks[k]), b->allocs.end());
        b->d_tasks[k] = nullptr;
    }
    b->ntasks[k] = (int)tasks.size();
    if (tasks.empty()) return LIBERI_OK;
    CUDA_TRY(cudaMalloc((void **)&b->d_tasks[k], tasks.size() * sizeof(int4)));
    b->allocs.push_back(b->d_tasks[k]);
    CUDA_TRY(cudaMemcpy(b->d_tasks[k], tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice));
    return LIBERI_OK;
}

static int batch_enqueue(liberi_batch b, cudaStream_t st, uint32_t mask) {
    liberi_handle h0 = b->hs[0];
    CUDA_TRY(launch_zero_fock(b->d_mols, (int)b->hs.size(), b->ntri_max, st));
    LaunchCtx ctx;
    ctx.basis = DevBasis{};
    ctx.rys_tab = h0->d_tab;
    ctx.rys_tabf = h0->d_tabf;
    ctx.Df = nullptr;
    ctx.D = nullptr;
    ctx.F = nullptr;
    ctx.schwarz_cut = h0->schwarz_cut;
    ctx.eri_cut = h0->eri_cut;
    ctx.stream = st;
    ctx.num_sms = h0->num_sms;
    const bool mixed = b->precision == 1;
    ctx.maxd = mixed ? b->d_maxd : nullptr;
    ctx.prim_cut = mixed ? b->fp32_prim * b->fp32_cut : 0.0;
    CUDA_TRY(launch_batch_prep(b->d_mols, (int)b->hs.size(), (long long)b->nbf_max * b->nbf_max,
                               mixed ? b->d_maxd : nullptr, st));
    if (!mixed) {
        for (int k = 0; k < NKERN; k++) {
            if (!((mask >> k) & 1u) || b->ntasks[k] == 0) continue;
            CUDA_TRY(launch_class_batch(k, ctx, b->d_tasks[k], b->ntasks[k], b->nbf_max, b->d_mols, b->d_cv[k],
                                        KDESC[k].swap, 0, nullptr));
        }
        return LIBERI_OK;
    }
    // mixed: every class's task split, then the FP64 lists on the side stream
    // beside the FP32 lists (as for single-molecule builds), joined back
    for (int k = 0; k < NKERN; k++) {
        if (!((mask >> k) & 1u) || b->ntasks[k] == 0) continue;
        CUDA_TRY(launch_split_batch(b->nitems[k], b->d_items[k], b->d_cv[k], b->d_maxd, b->fp32_cut, b->chunk[k],
                                    b->d_t64[k], b->d_t32[k], b->d_counts[k], st));
    }
    CUDA_TRY(cudaEventRecord(b->fork_ev, st));
    CUDA_TRY(cudaStreamWaitEvent(b->side, b->fork_ev, 0));
    for (int k = 0; k < NKERN; k++) {
        if (!((mask >> k) & 1u) || b->ntasks[k] == 0) continue;
        ctx.stream = b->side;
        CUDA_TRY(launch_class_batch(k, ctx, b->d_t64[k], b->cap[k], b->nbf_max, b->d_mols, b->d_cv[k],
                                    KDESC[k].swap, 0, b->d_counts[k]));
        ctx.stream = st;
        CUDA_TRY(launch_class_batch(k, ctx, b->d_t32[k], b->cap[k], b->nbf_max, b->d_mols, b->d_cv[k],
                                    KDESC[k].swap, 1, b->d_counts[k] + 1));
    }
    CUDA_TRY(cudaEventRecord(b->join_ev, b->side));
    CUDA_TRY(cudaStreamWaitEvent(st, b->join_ev, 0));
    return LIBERI_OK;
}

// ================================ C ABI ===========================================
extern "C" {

int liberi_c_last_error(char *buf, int32_t len) {
    if (!buf || len <= 0) return LIBERI_E_ARG;
    snprintf(buf, (size_t)len, "%s", g_err.c_str());
    return LIBERI_OK;
}

const char *liberi_c_kernel_name(int32_t k) { return (k >= 0 && k < NKALL) ? KDESC[k].name : nullptr; }

int liberi_c_rys_eval(int32_t n, double T, double thr, int32_t strict, double *u, double *w) {
    if (n < 1 || n > MAXROOT || !u || !w || !(T >= 0.0)) return fail(LIBERI_E_ARG, "liberi_rys_eval: bad argument");
    const std::vector<double> &tab = rys_table_host();
    const bool asym = strict ? (T > thr) : (T >= thr);
    if (asym || T >= RYS_TMAX) {
        const double it = 1.0 / T, sq = std::sqrt(it);
        for (int i = 0; i < n; i++) {
            u[i] = tab[rys_herm_off(n) + i] * it;
            w[i] = tab[rys_herm_off(n) + MAXROOT + i] * sq;
        }
        return LIBERI_OK;
    }
    const double t4 = T * (double)RYS_PER_UNIT;
    const int k = (int)t4;
    const double x = 2.0 * (t4 - (double)k) - 1.0;
    const double *base = tab.data() + rys_table_off(n) + (size_t)k * 2 * n * RYS_NCOEF;
    const double x2 = x * x, x4 = x2 * x2;
    for (int f = 0; f < 2 * n; f++) {  // same Estrin scheme as the device
        const double *c = base + f * RYS_NCOEF;
        const double a0 = std::fma(c[1], x, c[0]), a1 = std::fma(c[3], x, c[2]);
        const double a2 = std::fma(c[5], x, c[4]), a3 = std::fma(c[7], x, c[6]);
        const double b0 = std::fma(a1, x2, a0), b1 = std::fma(a3, x2, a2);
        const double v = std::fma(b1, x4, b0);
        if (f < n) u[f] = v; else w[f - n] = v;
    }
    return LIBERI_OK;
}

int liberi_c_rys7_eval(int32_t n, double T, double thr, int32_t strict, double *u, double *w) {
    if (n < 1 || n > MAXROOT7 || !u || !w || !(T >= 0.0)) return fail(LIBERI_E_ARG, "liberi_rys7_eval: bad argument");
    const std::vector<double> &tab = rys_table7_host();
    const bool asym = strict ? (T > thr) : (T >= thr);
    if (asym || T >= RYS7_TMAX) {
        const double it = 1.0 / T, sq = std::sqrt(it);
        for (int i = 0; i < n; i++) {
            u[i] = tab[rys7_herm_off(n) + i] * it;
            w[i] = tab[rys7_herm_off(n) + MAXROOT7 + i] * sq;
        }
        return LIBERI_OK;
    }
    const double t4 = T * (double)RYS_PER_UNIT;
    const int k = (int)t4;
    const double x = 2.0 * (t4 - (double)k) - 1.0, x2 = x * x, x4 = x2 * x2;
    const double *base = tab.data() + rys7_table_off(n) + (size_t)k * 2 * n * RYS_NCOEF;
    for (int f = 0; f < 2 * n; f++) {  // the f kernel's evaluation (k_f.cu rys7_root)
        const double *c = base + f * RYS_NCOEF;
        const double a0 = std::fma(c[1], x, c[0]), a1 = std::fma(c[3], x, c[2]);
        const double a2 = std::fma(c[5], x, c[4]), a3 = std::fma(c[7], x, c[6]);
        const double v = std::fma(std::fma(a3, x2, a2), x4, std::fma(a1, x2, a0));
        if (f < n) u[f] = v; else w[f - n] = v;
    }
    return LIBERI_OK;
}

int liberi_c_rys_eval_f32(int32_t n, float T, float thr, int32_t strict, float *u, float *w) {
    if (n < 1 || n > MAXROOT || !u || !w || !(T >= 0.0f)) return fail(LIBERI_E_ARG, "liberi_rys_eval_f32: bad argument");
    const std::vector<float> &tab = rys_table_f32_host();
    const bool asym = strict ? (T > thr) : (T >= thr);
    if (asym || T >= (float)RYS_TMAX) {
        const float it = 1.0f / T, sq = std::sqrt(it);
        for (int i = 0; i < n; i++) {
            u[i] = tab[rysf_herm_off(n) + i] * it;
            w[i] = tab[rysf_herm_off(n) + MAXROOT + i] * sq;
        }
        return LIBERI_OK;
    }
    const float t8 = T * (float)RYSF_PER_UNIT;
    const int k = (int)t8;
    const float x = 2.0f * (t8 - (float)k) - 1.0f;
    const float *base = tab.data() + rysf_table_off(n) + (size_t)k * 2 * n * RYSF_NCOEF;
    const float x2 = x * x;
    for (int f = 0; f < 2 * n; f++) {  // same evaluation as the device
        const float *c = base + f * RYSF_NCOEF;
        const float v = std::fmaf(std::fmaf(c[3], x, c[2]), x2, std::fmaf(c[1], x, c[0]));
        if (f < n) u[f] = v; else w[f - n] = v;
    }
    return LIBERI_OK;
}

int liberi_c_create(liberi_handle *handle) {
    if (!handle) return fail(LIBERI_E_ARG, "liberi_create: null handle pointer");
    *handle = new (std::nothrow) liberi_handle_s();
    if (!*handle) return fail(LIBERI_E_NOMEM, "liberi_create: out of host memory");
    memset(&(*handle)->stats, 0, sizeof(liberi_stats));
    return LIBERI_OK;
}

int liberi_c_cleanup(liberi_handle h) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_cleanup: null handle");
    if (!h->initialized) return LIBERI_OK;  // liberi_interface.F90:236
    DeviceGuard dev_guard(h->device);
    for (int k = 0; k <= NKERN; k++)
        for (int j = 0; j < 2; j++)
            if (h->ev[k][j]) {
                cudaEventDestroy(h->ev[k][j]);
                h->ev[k][j] = nullptr;
            }
    free_device(h);
    h->basis = BasisHost();
    h->pairs = PairsHost();
    h->initialized = false;
    return LIBERI_OK;
}

int liberi_c_destroy(liberi_handle h) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_destroy: null handle");
    liberi_c_cleanup(h);
    delete h;
    return LIBERI_OK;
}

int liberi_c_setup_bytes(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot, const int32_t *ang_mom,
                         const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                         const int32_t *atom_loc, const double *exponents, const double *contr_coef_s,
                         const double *contr_coef_p, const double *contr_coef_d, const double *contr_coef_f,
                         const double *coords, const double *schwrz_int, double schwarz_cut, int64_t *bytes) {
    if (!bytes) return fail(LIBERI_E_ARG, "liberi_setup_bytes: null result pointer");
    BasisHost b;
    int rc = copy_basis(b, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc, nullptr,
                        nullptr, exponents, contr_coef_s, contr_coef_p, contr_coef_d, contr_coef_f, coords,
                        schwrz_int);
    if (rc) return rc;
    rc = validate_basis(b);
    if (rc) return rc;
    PairsHost pr;
    std::vector<double4> shell_xyz;
    build_pairs(b, pr, shell_xyz);
    size_t total = basis_device_bytes(b, pr);
    std::vector<PlanHost> plans(NKALL);
    build_plans(pr, schwarz_cut, nullptr, 0, 0, 1, plans.data());
    for (int k = 0; k < NKALL; k++) total += plan_device_bytes(plans[k]);
    *bytes = (int64_t)total;
    return LIBERI_OK;
}

int liberi_c_setup(liberi_handle h, int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot,
                   const int32_t *ang_mom, const int32_t *contr_num, const int32_t *sh_loc,
                   const int32_t *atom_num, const int32_t *atom_loc, const int32_t *start_bas,
                   const int32_t *end_bas, const double *exponents, const double *contr_coef_s,
                   const double *contr_coef_p, const double *contr_coef_d, const double *contr_coef_f,
                   const double *coords, const double *schwrz_int, int32_t my_rank, int32_t num_procs) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_setup: null handle");
    if (num_procs < 1 || my_rank < 0 || my_rank >= num_procs)
        return fail(LIBERI_E_ARG, "liberi_setup: rank %d of %d is invalid", my_rank, num_procs);
    if (h->initialized) liberi_c_cleanup(h);  // liberi_interface.F90:134-136
    BasisHost b;
    int rc = copy_basis(b, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc,
                        start_bas, end_bas, exponents, contr_coef_s, contr_coef_p, contr_coef_d, contr_coef_f,
                        coords, schwrz_int);
    if (rc) return rc;
    rc = validate_basis(b);
    if (rc) return rc;
    if (h->max_device_bytes > 0.0) {
        // the caller's device-memory limit, from the host half of setup (the
        // same dry run as liberi_c_setup_bytes, with this handle's plan options)
        PairsHost pr;
        std::vector<double4> sx;
        build_pairs(b, pr, sx);
        size_t need = basis_device_bytes(b, pr);
        std::vector<PlanHost> plans(NKALL);
        build_plans(pr, h->schwarz_cut, h->chunk, h->rank_split, my_rank, num_procs, plans.data());
        for (int k = 0; k < NKALL; k++) need += plan_device_bytes(plans[k]);
        if ((double)need > h->max_device_bytes)
            return fail(LIBERI_E_NOMEM, "liberi_setup: needs %zu device bytes, above max_device_bytes = %.0f", need,
                        h->max_device_bytes);
    }
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, h->device));
    h->num_sms = prop.multiProcessorCount;
    h->basis = std::move(b);
    h->my_rank = my_rank;
    h->num_procs = num_procs;
    std::vector<double4> shell_xyz;
    build_pairs(h->basis, h->pairs, shell_xyz);
    // the handle's own stream at the highest priority: setup's kernels (the
    // primitive bounds) and copies then overtake the queued CTAs of builds
    // already running on the GPU (a serving loop sets sessions up while
    // others compute); builds through liberi_c_fock_build share it
    CUDA_TRY(high_priority_stream(&h->stream));
    rc = upload_basis(h, shell_xyz);
    if (!rc) rc = replan(h);
    if (rc) {
        free_device(h);
        return rc;
    }
    h->stats.device_bytes = (int64_t)h->dev.bytes;
    h->initialized = true;
    return LIBERI_OK;
}

int liberi_c_fock_build_device(liberi_handle h, const double *d_density, double *d_fock, void *stream) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_fock_build: null handle");
    if (!h->initialized) return fail(LIBERI_E_STATE, "liberi_fock_build called before liberi_setup");
    if (!d_density || !d_fock) return fail(LIBERI_E_ARG, "liberi_fock_build: null device buffer");
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    int rc = build_on_device(h, d_density, d_fock, st);
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return LIBERI_OK;
}

int liberi_c_fock_build_uhf_device(liberi_handle h, const double *d_density_a, const double *d_density_b,
                                   double *d_fock_a, double *d_fock_b, void *stream) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_fock_build_uhf: null handle");
    if (!h->initialized) return fail(LIBERI_E_STATE, "liberi_fock_build_uhf called before liberi_setup");
    if (!d_density_a || !d_density_b || !d_fock_a || !d_fock_b)
        return fail(LIBERI_E_ARG, "liberi_fock_build_uhf: null device buffer");
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    int rc = build_on_device(h, d_density_a, d_fock_a, st, d_density_b, 0);
    if (!rc) rc = build_on_device(h, d_density_a, d_fock_b, st, d_density_b, 1);
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return LIBERI_OK;
}

int liberi_c_fock_build_uhf(liberi_handle h, const double *density_a, const double *density_b, double *fock_a,
                            double *fock_b, int32_t matrix_size) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_fock_build_uhf: null handle");
    if (!h->initialized) return fail(LIBERI_E_STATE, "liberi_fock_build_uhf called before liberi_setup");
    const long long n = h->basis.num_bas;
    if ((long long)matrix_size != n * (n + 1) / 2)
        return fail(LIBERI_E_SIZE, "liberi_fock_build_uhf: matrix_size %d != num_bas(num_bas+1)/2 = %lld",
                    matrix_size, n * (n + 1) / 2);
    if (!density_a || !density_b || !fock_a || !fock_b) return fail(LIBERI_E_ARG, "liberi_fock_build_uhf: null buffer");
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaStream_t st = h->stream;
    const size_t bytes = (size_t)matrix_size * sizeof(double);
    // the beta density and Fock matrix in a stream-ordered scratch pair beside the handle's own D and F
    double *db = nullptr, *fb = nullptr;
    CUDA_TRY(cudaMallocAsync((void **)&db, 2 * bytes, st));
    fb = db + matrix_size;
    cudaError_t e = cudaMemcpyAsync(h->dev.D, density_a, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, density_b, bytes, cudaMemcpyHostToDevice, st);
    int rc = LIBERI_OK;
    if (e == cudaSuccess) {
        rc = build_on_device(h, h->dev.D, h->dev.F, st, db, 0);
        if (!rc) rc = build_on_device(h, h->dev.D, fb, st, db, 1);
    }
    if (e == cudaSuccess && !rc) e = cudaMemcpyAsync(fock_a, h->dev.F, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && !rc) e = cudaMemcpyAsync(fock_b, fb, bytes, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(db, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc) return rc;
    CUDA_TRY(e);
    return LIBERI_OK;
}

int liberi_c_fock_build(liberi_handle h, const double *density, double *fock, int32_t matrix_size) {
    if (!h) return fail(LIBERI_E_ARG, "liberi_fock_build: null handle");
    if (!h->initialized) return fail(LIBERI_E_STATE, "liberi_fock_build called before liberi_setup");
    const long long n = h->basis.num_bas;
    if ((long long)matrix_size != n * (n + 1) / 2)
        return fail(LIBERI_E_SIZE, "liberi_fock_build: matrix_size %d != num_bas(num_bas+1)/2 = %lld",
                    matrix_size, n * (n + 1) / 2);
    if (!density || !fock) return fail(LIBERI_E_ARG, "liberi_fock_build: null buffer");
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaStream_t st = h->stream;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, st));
    CUDA_TRY(cudaMemcpyAsync(h->dev.D, density, (size_t)matrix_size * sizeof(double), cudaMemcpyHostToDevice, st));
    int rc = build_on_device(h, h->dev.D, h->dev.F, st);
    if (rc) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(fock, h->dev.F, (size_t)matrix_size * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaEventRecord(e1, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    h->stats.build_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return LIBERI_OK;
}

int liberi_c_batch_create(liberi_batch *out, const liberi_handle *handles, int32_t n) {
    if (!out || !handles || n <= 0) return fail(LIBERI_E_ARG, "liberi_batch_create: bad arguments");
    liberi_batch b = new (std::nothrow) liberi_batch_s();
    if (!b) return fail(LIBERI_E_NOMEM, "liberi_batch_create: out of host memory");
    for (int i = 0; i < n; i++) {
        liberi_handle h = handles[i];
        if (!h || !h->initialized) {
            delete b;
            return fail(LIBERI_E_STATE, "liberi_batch_create: handle %d is not set up", i);
        }
        if (h->num_procs != 1 || h->device != handles[0]->device || h->precision != handles[0]->precision ||
            h->schwarz_cut != handles[0]->schwarz_cut || h->eri_cut != handles[0]->eri_cut ||
            (h->precision == 1 && (h->fp32_cut != handles[0]->fp32_cut || h->fp32_prim != handles[0]->fp32_prim))) {
            delete b;
            return fail(LIBERI_E_ARG, "liberi_batch_create: handle %d differs in device, rank split, precision or cuts", i);
        }
        if (h->pairs.nl[3] > 0) {
            delete b;
            return fail(LIBERI_E_UNSUPPORTED, "liberi_batch_create: handle %d has f shells; batched builds cover s/p/d", i);
        }
        if (h->plan_dirty) {
            int rc = replan(h);
            if (rc) {
                delete b;
                return rc;
            }
        }
        b->hs.push_back(h);
        b->nbf_max = std::max(b->nbf_max, h->basis.num_bas);
    }
    b->ntri_max = (long long)b->nbf_max * (b->nbf_max + 1) / 2;
    b->device = handles[0]->device;
    DeviceGuard dev_guard(b->device);
    int rc = LIBERI_OK;
    auto die = [&](int code) { batch_free(b); delete b; return code; };
    if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join_ev, cudaEventDisableTiming) != cudaSuccess)
        return die(fail(LIBERI_E_DEVICE, "liberi_batch_create: stream or event creation failed"));
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return die(fail(LIBERI_E_DEVICE, "liberi_batch_create: stream creation failed"));
    if (cudaMalloc((void **)&b->d_mols, n * sizeof(MolView)) != cudaSuccess)
        return die(fail(LIBERI_E_NOMEM, "liberi_batch_create: out of device memory"));
    b->allocs.push_back(b->d_mols);
    for (int k = 0; k < NKERN; k++) {
        std::vector<ClassView> cv(n);
        for (int m = 0; m < n; m++)
            cv[m] = ClassView{b->hs[m]->plan[k].d_bra, b->hs[m]->plan[k].d_ket, b->hs[m]->plan[k].d_bra_x,
                              b->hs[m]->plan[k].d_ket_x, b->hs[m]->plan[k].d_ket_rec};
        if (cudaMalloc((void **)&b->d_cv[k], n * sizeof(ClassView)) != cudaSuccess)
            return die(fail(LIBERI_E_NOMEM, "liberi_batch_create: out of device memory"));
        b->allocs.push_back(b->d_cv[k]);
        cudaMemcpy(b->d_cv[k], cv.data(), n * sizeof(ClassView), cudaMemcpyHostToDevice);
        b->chunk[k] = default_chunk(k);
        rc = batch_build_tasks(b, k);
        if (rc) return die(rc);
    }
    b->precision = handles[0]->precision;
    b->fp32_cut = handles[0]->fp32_cut;
    b->fp32_prim = handles[0]->fp32_prim;
    {  // every molecule's D as a full matrix, made per iteration from its packed D
        size_t sqtot = 0;
        for (int m = 0; m < n; m++) {
            b->sq_off.push_back(sqtot);
            const size_t nb = (size_t)b->hs[m]->basis.num_bas;
            sqtot += nb * nb;
        }
        if (cudaMalloc((void **)&b->d_Dsq, std::max<size_t>(sqtot, 1) * sizeof(double)) != cudaSuccess)
            return die(fail(LIBERI_E_NOMEM, "liberi_batch_create: out of device memory"));
        b->allocs.push_back(b->d_Dsq);
        if (b->precision == 1) {
            if (cudaMalloc((void **)&b->d_Df, std::max<size_t>(sqtot, 1) * sizeof(float)) != cudaSuccess)
                return die(fail(LIBERI_E_NOMEM, "liberi_batch_create: out of device memory"));
            b->allocs.push_back(b->d_Df);
        }
    }
    if (b->precision == 1) {
        // every molecule's items of a class in one list; task capacity for the
        // smallest kets-per-task the tuner may choose
        if (cudaMalloc((void **)&b->d_maxd, n * sizeof(unsigned long long)) != cudaSuccess)
            return die(fail(LIBERI_E_NOMEM, "liberi_batch_create: out of device memory"));
        b->allocs.push_back(b->d_maxd);
        for (int k = 0; k < NKERN; k++) {
            std::vector<int4> items;
            long long cap = 0;
            for (int m = 0; m < n; m++)
                for (const int4 &it : b->hs[m]->plan[k].items) {
                    items.push_back(make_int4(it.x, it.y, it.z, m));
                    cap += (it.z + TUNE_CHUNKS[0] - 1) / TUNE_CHUNKS[0] + 1;
                }
            if (items.empty()) continue;
            if (cap > INT32_MAX) return die(fail(LIBERI_E_UNSUPPORTED, "liberi_batch_create: batch too large"));
            b->nitems[k] = (int)items.size();
            b->cap[k] = (int)cap;
            if (cudaMalloc((void **)&b->d_items[k], items.size() * sizeof(int4)) != cudaSuccess ||
                cudaMalloc((void **)&b->d_t64[k], cap * sizeof(int4)) != cudaSuccess ||
                cudaMalloc((void **)&b->d_t32[k], cap * sizeof(int4)) != cudaSuccess ||
                cudaMalloc((void **)&b->d_counts[k], 4 * sizeof(int)) != cudaSuccess)
                return die(fail(LIBERI_E_NOMEM, "liberi_batch_create: out of device memory"));
            for (void *p : {(void *)b->d_items[k], (void *)b->d_t64[k], (void *)b->d_t32[k], (void *)b->d_counts[k]})
                b->allocs.push_back(p);
            cudaMemcpy(b->d_items[k], items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice);
        }
    }
    *out = b;
    return LIBERI_OK;
}

int liberi_c_batch_bind(liberi_batch b, const double *const *d_density, double *const *d_fock) {
    if (!b || !d_density || !d_fock) return fail(LIBERI_E_ARG, "liberi_batch_bind: null argument");
    DeviceGuard dev_guard(b->device);
    CUDA_TRY(dev_guard.err);
    std::vector<MolView> mv(b->hs.size());
    for (size_t m = 0; m < b->hs.size(); m++) {
        if (!d_density[m] || !d_fock[m]) return fail(LIBERI_E_ARG, "liberi_batch_bind: null buffer %zu", m);
        mv[m].b = dev_basis(b->hs[m]);
        mv[m].D = d_density[m];
        mv[m].Dsq = b->d_Dsq + b->sq_off[m];
        mv[m].F = d_fock[m];
        mv[m].Df = b->precision == 1 ? b->d_Df + b->sq_off[m] : nullptr;
        mv[m].nbf = b->hs[m]->basis.num_bas;
        mv[m].pad = 0;
    }
    // a captured graph reads the views through d_mols, so rebinding needs no re-capture
    CUDA_TRY(cudaMemcpy(b->d_mols, mv.data(), mv.size() * sizeof(MolView), cudaMemcpyHostToDevice));
    b->bound = true;
    return LIBERI_OK;
}

int liberi_c_batch_fock_build(liberi_batch b, void *stream) {
    if (!b) return fail(LIBERI_E_ARG, "liberi_batch_fock_build: null batch");
    if (!b->bound) return fail(LIBERI_E_STATE, "liberi_batch_fock_build: call liberi_c_batch_bind first");
    DeviceGuard dev_guard(b->device);
    CUDA_TRY(dev_guard.err);
    return batch_enqueue(b, stream ? (cudaStream_t)stream : b->stream, (1u << NKERN) - 1);
}

int liberi_c_batch_capture(liberi_batch b) {
    if (!b) return fail(LIBERI_E_ARG, "liberi_batch_capture: null batch");
    if (!b->bound) return fail(LIBERI_E_STATE, "liberi_batch_capture: call liberi_c_batch_bind first");
    DeviceGuard dev_guard(b->device);
    CUDA_TRY(dev_guard.err);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    // attributes set outside capture (dynamic shared memory of each class)
    int rc = batch_enqueue(b, b->stream, (1u << NKERN) - 1);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    rc = batch_enqueue(b, b->stream, (1u << NKERN) - 1);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(LIBERI_E_DEVICE, "liberi_batch_capture: %s", cudaGetErrorString(e));
    b->graph = g;
    CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return LIBERI_OK;
}

int liberi_c_batch_launch(liberi_batch b, void *stream) {
    if (!b || !b->exec) return fail(LIBERI_E_STATE, "liberi_batch_launch: no captured graph");
    DeviceGuard dev_guard(b->device);
    CUDA_TRY(dev_guard.err);
    CUDA_TRY(cudaGraphLaunch(b->exec, stream ? (cudaStream_t)stream : b->stream));
    return LIBERI_OK;
}

int liberi_c_batch_synchronize(liberi_batch b) {
    if (!b) return fail(LIBERI_E_ARG, "liberi_batch_synchronize: null batch");
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return LIBERI_OK;
}

int liberi_c_batch_destroy(liberi_batch b) {
    if (!b) return fail(LIBERI_E_ARG, "liberi_batch_destroy: null batch");
    DeviceGuard dev_guard(b->device);
    batch_free(b);
    delete b;
    return LIBERI_OK;
}

// ---- autotuner: kets per CTA task, per class ------------------------------------

int liberi_c_batch_autotune(liberi_batch b, int32_t reps, int32_t *chunks_out) {
    if (!b || !b->bound) return fail(LIBERI_E_STATE, "liberi_batch_autotune: batch not bound");
    if (reps < 1) reps = 1;
    DeviceGuard dev_guard(b->device);
    CUDA_TRY(dev_guard.err);
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    for (int k = 0; k < NKERN; k++) {
        long long work = 0;
        for (auto h : b->hs) work += h->plan[k].total;
        if (work == 0) continue;
        float best = 1e30f;
        int best_c = b->chunk[k];
        for (int c : TUNE_CHUNKS) {
            b->chunk[k] = c;
            int rc = batch_build_tasks(b, k);
            if (rc) return rc;
            rc = batch_enqueue(b, b->stream, 1u << k);  // warm-up
            if (rc) return rc;
            CUDA_TRY(cudaEventRecord(e0, b->stream));
            for (int r = 0; r < reps; r++) {
                rc = batch_enqueue(b, b->stream, 1u << k);
                if (rc) return rc;
            }
            CUDA_TRY(cudaEventRecord(e1, b->stream));
            CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                best_c = c;
            }
        }
        b->chunk[k] = best_c;
        int rc = batch_build_tasks(b, k);
        if (rc) return rc;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (chunks_out)
        for (int k = 0; k < NKERN; k++) chunks_out[k] = b->chunk[k];
    if (b->exec) return liberi_c_batch_capture(b);  // re-capture with the tuned tasks
    return LIBERI_OK;
}

int liberi_c_autotune(liberi_handle h, int32_t reps, int32_t *chunks_out) {
    if (!h || !h->initialized) return fail(LIBERI_E_STATE, "liberi_autotune: handle not set up");
    if (reps < 1) reps = 1;
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    const uint32_t mask0 = h->class_mask;
    const int prec0 = h->precision;
    const double cut0 = h->fp32_cut;
    int rc = LIBERI_OK;
    // time one configuration of class k: reps builds of that class alone
    auto time_class = [&](int k, float *ms) -> int {
        h->class_mask = 1u << k;
        int r = build_on_device(h, h->dev.D, h->dev.F, h->stream);  // warm-up
        if (r) return r;
        cudaEventRecord(e0, h->stream);
        for (int i = 0; i < reps && !r; i++) r = build_on_device(h, h->dev.D, h->dev.F, h->stream);
        cudaEventRecord(e1, h->stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms, e0, e1);
        return r;
    };
    for (int k = 0; k < NKERN && !rc; k++) {
        if (h->plan_dirty) rc = replan(h);
        if (rc || h->plan[k].total == 0) continue;
        // FP64: shape variant x kets per task
        h->precision = 0;
        float best = 1e30f;
        int best_c = h->plan[k].chunk, best_v = h->variant[0][k];
        for (int v = 0; v < NVARIANT && !rc; v++) {
            h->variant[0][k] = v;
            for (int c : TUNE_CHUNKS) {
                PlanHost &ph = h->plan[k];
                ph.chunk = c;
                ph.tasks.clear();
                make_tasks(ph, c, 0, ph.tasks);
                if (ph.d_tasks) {  // used only by this tuner's builds on the handle's stream
                    dev_release(h, ph.d_tasks);
                    ph.d_tasks = nullptr;
                }
                if (dev_upload(h, &ph.d_tasks, ph.tasks.data(), ph.tasks.size()) != cudaSuccess) {
                    rc = fail(LIBERI_E_NOMEM, "liberi_autotune: out of device memory");
                    break;
                }
                float ms = 0.f;
                rc = time_class(k, &ms);
                if (rc) break;
                if (ms < best) {
                    best = ms;
                    best_c = c;
                    best_v = v;
                }
            }
        }
        if (rc) break;
        h->chunk[k] = best_c;
        h->variant[0][k] = best_v;
        // FP32 tier shape (handles in mixed precision), timed on the class's
        // build at the handle's own cut (its FP32 primitive screening follows
        // the cut: a cut that sent every quartet to FP32 would skip every
        // primitive)
        if (prec0 == 1) {
            h->precision = 1;
            h->fp32_cut = cut0;
            float best32 = 1e30f;
            int best_v32 = h->variant[1][k];
            for (int v = 0; v < NVARIANT && !rc; v++) {
                h->variant[1][k] = v;
                float ms = 0.f;
                rc = time_class(k, &ms);
                if (!rc && ms < best32) {
                    best32 = ms;
                    best_v32 = v;
                }
            }
            h->variant[1][k] = best_v32;
            h->fp32_cut = cut0;
        }
    }
    h->class_mask = mask0;
    h->precision = prec0;
    h->fp32_cut = cut0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    h->plan_dirty = true;  // rebuild plans with the tuned chunks on the next build
    rc = replan(h);
    if (chunks_out)
        for (int k = 0; k < NKERN; k++) chunks_out[k] = h->plan[k].chunk;
    return rc;
}

int liberi_c_set_class_variant(liberi_handle h, int32_t k, int32_t precision, int32_t variant) {
    if (!h || k < 0 || k >= NKERN || precision < 0 || precision > 1 || variant < 0 || variant >= NVARIANT)
        return fail(LIBERI_E_ARG, "liberi_set_class_variant: bad argument");
    h->variant[precision][k] = variant;
    return LIBERI_OK;
}

int liberi_c_get_class_variant(liberi_handle h, int32_t k, int32_t precision, int32_t *variant) {
    if (!h || !variant || k < 0 || k >= NKERN || precision < 0 || precision > 1)
        return fail(LIBERI_E_ARG, "liberi_get_class_variant: bad argument");
    *variant = h->variant[precision][k];
    return LIBERI_OK;
}

int liberi_c_set_option(liberi_handle h, const char *name, double value) {
    if (!h || !name) return fail(LIBERI_E_ARG, "liberi_set_option: null argument");
    std::string n(name);
    if (n == "schwarz_cut") {
        if (!(value > 0)) return fail(LIBERI_E_ARG, "schwarz_cut must be > 0");
        h->schwarz_cut = value;
        h->plan_dirty = h->initialized;
    } else if (n == "eri_cut") {
        if (!(value >= 0)) return fail(LIBERI_E_ARG, "eri_cut must be >= 0");
        h->eri_cut = value;
    } else if (n == "fp32_cut") {
        if (!(value >= 0)) return fail(LIBERI_E_ARG, "fp32_cut must be >= 0");
        h->fp32_cut = value;
    } else if (n == "max_device_bytes") {
        if (!(value >= 0)) return fail(LIBERI_E_ARG, "max_device_bytes must be >= 0");
        h->max_device_bytes = value;
    } else if (n == "fp32_prim") {
        if (!(value >= 0 && value <= 1)) return fail(LIBERI_E_ARG, "fp32_prim must be in [0, 1]");
        h->fp32_prim = value;
    } else if (n == "precision") {
        if (value != 0 && value != 1) return fail(LIBERI_E_ARG, "precision must be 0 or 1");
        h->precision = (int)value;
    } else if (n == "device") {
        if (h->initialized) return fail(LIBERI_E_STATE, "device must be chosen before setup");
        h->device = (int)value;
    } else if (n == "class_mask") {
        if (!(value >= 0 && value < (double)(1u << NKERN))) return fail(LIBERI_E_ARG, "class_mask out of range");
        h->class_mask = (uint32_t)value;
    } else if (n == "rank_split") {
        if (value != 0 && value != 1) return fail(LIBERI_E_ARG, "rank_split must be 0 or 1");
        if (h->initialized) return fail(LIBERI_E_STATE, "rank_split must be chosen before setup");
        h->rank_split = (int)value;
    } else if (n == "side_mask") {
        if (!(value >= 0 && value < (double)(1u << NKERN))) return fail(LIBERI_E_ARG, "side_mask out of range");
        h->side_mask = (uint32_t)value;
    } else if (n == "overlap") {
        h->overlap = value != 0;
    } else if (n == "fan") {
        h->fan_out = value != 0;
    } else if (n == "tile_mask") {
        if (!(value >= 0 && value < (double)(1u << NKERN))) return fail(LIBERI_E_ARG, "tile_mask out of range");
        h->tile_mask = (uint32_t)value;
    } else if (n == "timing") {
        h->timing = value != 0;
    } else {
        return fail(LIBERI_E_ARG, "unknown option '%s'", name);
    }
    return LIBERI_OK;
}

int liberi_c_get_option(liberi_handle h, const char *name, double *value) {
    if (!h || !name || !value) return fail(LIBERI_E_ARG, "liberi_get_option: null argument");
    std::string n(name);
    if (n == "schwarz_cut") *value = h->schwarz_cut;
    else if (n == "eri_cut") *value = h->eri_cut;
    else if (n == "fp32_cut") *value = h->fp32_cut;
    else if (n == "fp32_prim") *value = h->fp32_prim;
    else if (n == "max_device_bytes") *value = h->max_device_bytes;
    else if (n == "precision") *value = h->precision;
    else if (n == "device") *value = h->device;
    else if (n == "class_mask") *value = h->class_mask;
    else if (n == "tile_mask") *value = h->tile_mask;
    else if (n == "side_mask") *value = h->side_mask;
    else if (n == "overlap") *value = h->overlap ? 1 : 0;
    else if (n == "fan") *value = h->fan_out ? 1 : 0;
    else if (n == "rank_split") *value = h->rank_split;
    else if (n == "timing") *value = h->timing ? 1 : 0;
    else return fail(LIBERI_E_ARG, "unknown option '%s'", name);
    return LIBERI_OK;
}

int liberi_c_get_stats(liberi_handle h, liberi_stats *stats) {
    if (!h || !stats) return fail(LIBERI_E_ARG, "liberi_get_stats: null argument");
    for (int k = 0; k < NKERN; k++) {
        h->stats.fp32_quartets[k] = 0;
        if (h->initialized && h->precision == 1 && h->plan[k].d_ntasks) {
            int cnt[4] = {0, 0, 0, 0};
            if (cudaMemcpy(cnt, h->plan[k].d_ntasks, sizeof(cnt), cudaMemcpyDeviceToHost) == cudaSuccess)
                h->stats.fp32_quartets[k] = (int64_t)(unsigned)cnt[2] | ((int64_t)(unsigned)cnt[3] << 32);
        }
    }
    for (int k = 0; k < NKERN; k++) {
        h->stats.kernel_ms[k] = 0.0;
        if (h->timing && h->ev_recorded[k]) {
            float ms = 0.f;
            if (cudaEventSynchronize(h->ev[k][1]) == cudaSuccess &&
                cudaEventElapsedTime(&ms, h->ev[k][0], h->ev[k][1]) == cudaSuccess)
                h->stats.kernel_ms[k] = ms;
        }
    }
    *stats = h->stats;
    return LIBERI_OK;
}

int liberi_c_get_class_stats(liberi_handle h, int32_t k, int64_t *out) {
    if (!h || !out || k < 0 || k >= NKALL) return fail(LIBERI_E_ARG, "liberi_get_class_stats: bad argument");
    out[0] = k < NKERN ? h->stats.quartets[k] : h->fq[k - NKERN];
    out[1] = k < NKERN ? h->stats.prim_quartets[k] : h->fprim[k - NKERN];
    return LIBERI_OK;
}

// {count, sum, xor} per class for classes 0..nclass-1 (see the header)
static int quartet_fingerprint(liberi_handle h, int nclass, uint64_t *out) {
    if (!h || !out) return fail(LIBERI_E_ARG, "liberi_quartet_fingerprint: null argument");
    if (!h->initialized) return fail(LIBERI_E_STATE, "liberi_quartet_fingerprint called before liberi_setup");
    if (h->plan_dirty) return fail(LIBERI_E_STATE, "liberi_quartet_fingerprint: options changed since the last build");
    DeviceGuard dev_guard(h->device);
    CUDA_TRY(dev_guard.err);
    cudaStream_t st = h->stream;
    unsigned long long *d_out = nullptr;
    CUDA_TRY(cudaMallocAsync((void **)&d_out, 3 * NKALL * sizeof(unsigned long long), st));
    cudaError_t e = cudaMemsetAsync(d_out, 0, 3 * NKALL * sizeof(unsigned long long), st);
    LaunchCtx ctx{};
    ctx.basis = dev_basis(h);
    ctx.stream = st;
    for (int k = 0; k < nclass && e == cudaSuccess; k++) {
        const PlanHost &ph = h->plan[k];
        if (ph.total == 0 || (k < NKERN && !((h->class_mask >> k) & 1u))) continue;
        const RankSplit rs = rank_split_of(h, k);
        DevPlan dp = dev_plan_of(h, k);
        if (!h->last_split_lists || k >= NKERN) {  // f classes: always the static FP64 list
            e = launch_quartet_fp(k, ctx, dp, rs, d_out + 3 * k);
            continue;
        }
        // the lists the last (mixed-precision) build split and launched
        dp.ntasks = ph.task_cap;
        dp.tasks = ph.d_tasks64;
        dp.ntasks_dev = ph.d_ntasks;
        e = launch_quartet_fp(k, ctx, dp, rs, d_out + 3 * k);
        if (e != cudaSuccess) break;
        dp.tasks = ph.d_tasks32;
        dp.ntasks_dev = ph.d_ntasks + 1;
        e = launch_quartet_fp(k, ctx, dp, rs, d_out + 3 * k);
    }
    unsigned long long host[3 * NKALL];
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d_out, sizeof(host), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d_out, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    CUDA_TRY(e);
    for (int i = 0; i < 3 * nclass; i++) out[i] = host[i];
    return LIBERI_OK;
}

int liberi_c_quartet_fingerprint(liberi_handle h, uint64_t *out) { return quartet_fingerprint(h, NKERN, out); }

int liberi_c_quartet_fingerprint_all(liberi_handle h, uint64_t *out) { return quartet_fingerprint(h, NKALL, out); }

int liberi_c_schwarz(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot, const int32_t *ang_mom,
                     const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                     const int32_t *atom_loc, const double *exponents, const double *contr_coef_s,
                     const double *contr_coef_p, const double *contr_coef_d, const double *contr_coef_f,
                     const double *coords, double *schwrz_out) {
    if (!schwrz_out) return fail(LIBERI_E_ARG, "liberi_schwarz: null output");
    liberi_handle_s tmp;
    std::vector<double> ones((size_t)(nsh > 0 ? nsh : 0) * (nsh + 1) / 2, 1.0);
    int rc = copy_basis(tmp.basis, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num,
                        atom_loc, nullptr, nullptr, exponents, contr_coef_s, contr_coef_p, contr_coef_d,
                        contr_coef_f, coords, ones.data());
    if (rc) return rc;
    rc = validate_basis(tmp.basis);
    if (rc) return rc;
    CUDA_TRY(cudaGetDevice(&tmp.device));  // the caller's current device
    std::vector<double4> shell_xyz;
    build_pairs(tmp.basis, tmp.pairs, shell_xyz);
    CUDA_TRY(high_priority_stream(&tmp.stream));
    rc = upload_basis(&tmp, shell_xyz);
    double *d_out = nullptr;
    const int npairs = tmp.pairs.class_off[NPC];
    if (!rc) {
        cudaError_t e = dev_alloc(&tmp, &d_out, (size_t)npairs);
        if (e != cudaSuccess) rc = fail(LIBERI_E_NOMEM, "liberi_schwarz: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        DevBasis db = dev_basis(&tmp);
        for (int c = 0; c < NPC && !rc; c++) {
            int off = tmp.pairs.class_off[c], n = tmp.pairs.class_off[c + 1] - off;
            // s/p/d pair classes by their Rys kernels, f ones by the f classes' evaluation
            cudaError_t e = c < NPC_SPD ? launch_schwarz(c, n, off, db, tmp.d_tab, d_out + off, tmp.stream)
                                        : launch_fschwarz(c, n, off, db, tmp.d_tab7, d_out, tmp.stream);
            if (e != cudaSuccess) rc = fail(LIBERI_E_DEVICE, "liberi_schwarz: %s", cudaGetErrorString(e));
        }
    }
    std::vector<double> per_pair(npairs);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(per_pair.data(), d_out, npairs * sizeof(double), cudaMemcpyDeviceToHost,
                                        tmp.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(tmp.stream);
        if (e != cudaSuccess) rc = fail(LIBERI_E_DEVICE, "liberi_schwarz: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        const size_t ntri = (size_t)nsh * (nsh + 1) / 2;
        std::fill(schwrz_out, schwrz_out + ntri, 0.0);
        for (int p = 0; p < npairs; p++) {
            int hi = std::max(tmp.pairs.ish[p], tmp.pairs.jsh[p]) + 1, lo = std::min(tmp.pairs.ish[p], tmp.pairs.jsh[p]) + 1;
            schwrz_out[(size_t)hi * (hi - 1) / 2 + lo - 1] = per_pair[p];
        }
    }
    free_device(&tmp);
    return rc;
}

// ---- GAMESS direct-link wrapper (module-level saved handle) ------------------------
static std::mutex g_wrap_mu;
static liberi_handle g_wrap = nullptr;
static long long g_wrap_size = 0;

int liberi_c_init(int32_t natoms, int32_t num_bas, int32_t nsh, int32_t mxgtot, const int32_t *ang_mom,
                  const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                  const int32_t *atom_loc, const int32_t *start_bas, const int32_t *end_bas,
                  const double *exponents, const double *contr_coef_s, const double *contr_coef_p,
                  const double *contr_coef_d, const double *contr_coef_f, const double *coords,
                  const double *schwrz_int, int32_t my_rank, int32_t num_procs) {
    std::lock_guard<std::mutex> lk(g_wrap_mu);
    if (g_wrap) {  // gms_liberi_wrapper.F90:82-85
        liberi_c_cleanup(g_wrap);
        liberi_c_destroy(g_wrap);
        g_wrap = nullptr;
    }
    int rc = liberi_c_create(&g_wrap);
    if (rc) return rc;
    rc = liberi_c_setup(g_wrap, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc,
                        start_bas, end_bas, exponents, contr_coef_s, contr_coef_p, contr_coef_d, contr_coef_f,
                        coords, schwrz_int, my_rank, num_procs);
    if (rc) {
        std::string msg = g_err;
        liberi_c_destroy(g_wrap);
        g_wrap = nullptr;
        g_err = msg;
        return rc;
    }
    g_wrap_size = (long long)num_bas * (num_bas + 1) / 2;
    return LIBERI_OK;
}

int liberi_c_fock(const double *density, double *fock, int32_t n) {
    std::lock_guard<std::mutex> lk(g_wrap_mu);
    if (!g_wrap) return fail(LIBERI_E_STATE, "liberi_fock called before liberi_init");
    if ((long long)n != g_wrap_size)  // gms_liberi_wrapper.F90:122-127
        return fail(LIBERI_E_SIZE, "matrix size mismatch in liberi_fock: expected %lld, got %d", g_wrap_size, n);
    return liberi_c_fock_build(g_wrap, density, fock, n);
}

int liberi_c_finalize(void) {
    std::lock_guard<std::mutex> lk(g_wrap_mu);
    if (g_wrap) {
        liberi_c_cleanup(g_wrap);
        liberi_c_destroy(g_wrap);
        g_wrap = nullptr;
    }
    return LIBERI_OK;
}

}  // extern "C"
