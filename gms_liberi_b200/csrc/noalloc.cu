// noalloc.cu -- Schwarz-table generator that allocates no device memory.
//
// liberi_c_schwarz obtains its device working memory (device copies of the
// shell, pair and primitive-pair data, the Rys tables and one result per
// pair) with cudaMalloc on every call.  Some callers cannot do that: a host
// program that has already handed nearly all of the GPU's memory to its own
// pool allocator (an SCF driver that sized its buffers at start-up, where a
// late cudaMalloc fails or fragments the pool), or one whose allocation
// policy forbids ad-hoc cudaMalloc/cudaFree because they synchronise the
// device behind its back.  liberi_c_schwarz_noalloc gives them the same
// table from a fixed, file-scope device array instead.
//
// Contract:
//   * LIBERI_NOALLOC_SCRATCH_BYTES (8 MiB) of device memory is held by every
//     GPU on which this entry point has run, until process exit.  CUDA loads
//     a library's device code lazily by default, so the array is committed
//     by the first call on each device, not when the library is loaded: a
//     caller whose pool will claim nearly all of the GPU's memory should make
//     one call per device at start-up, before the pool does.  If that first
//     call cannot get the memory it fails with LIBERI_E_NOMEM;
//   * the first call on a device also loads the module, so it should come
//     before any stream capture on that device;
//   * bases whose device data does not fit are rejected (LIBERI_E_NOMEM, the
//     message states the bytes needed and the limit) before any GPU work;
//   * no cudaMalloc, cudaFree or other allocating routine is called; work
//     runs on the legacy default stream and the call returns after the
//     results have been copied back;
//   * every call reuses the same array, which keeps the previous call's
//     contents: the Rys tables are copied in and the result region is
//     cleared on every call.  Calls are serialised by a process-wide lock;
//     uses of the array that overlap on the GPU (from code that bypasses this
//     entry point) would race.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/liberi_b200.h"
#include "engine.h"

namespace liberi {
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)LIBERI_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// With the caller's device current: the array's device address (the host-side
// symbol is only a stand-in) and the Rys tables copied into its head.  The
// address is looked up on every call, never cached: a context that was
// destroyed and re-created (cudaDeviceReset) gets a new module instance whose
// array may sit elsewhere and holds no tables.  Once the module is loaded the
// lookup allocates nothing; the table copy is 0.46 MB.
int setup_device(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        // the first use on a device loads the module and commits the array
        const int code = e == cudaErrorMemoryAllocation ? LIBERI_E_NOMEM : LIBERI_E_DEVICE;
        return set_error(code, (std::string("liberi_schwarz_noalloc: cudaGetSymbolAddress failed: ") +
                                cudaGetErrorString(e)).c_str());
    }
    const std::vector<double> &tab = rys_table_host();
    e = cudaMemcpy(p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
        return set_error(LIBERI_E_DEVICE, (std::string("liberi_schwarz_noalloc: table upload failed: ") +
                                           cudaGetErrorString(e)).c_str());
    *out = (unsigned char *)p;
    return LIBERI_OK;
}

}  // namespace
}  // namespace liberi

using namespace liberi;

extern "C" int liberi_c_schwarz_noalloc(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot,
                                        const int32_t *ang_mom, const int32_t *contr_num, const int32_t *sh_loc,
                                        const int32_t *atom_num, const int32_t *atom_loc, const double *exponents,
                                        const double *contr_coef_s, const double *contr_coef_p,
                                        const double *contr_coef_d, const double *coords, double *schwrz_out) {
    if (!schwrz_out) return set_error(LIBERI_E_ARG, "liberi_schwarz_noalloc: null output");
    BasisHost basis;
    PairsHost pairs;
    std::vector<double4> shell_xyz;
    int rc = schwarz_host_inputs(nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc,
                                 exponents, contr_coef_s, contr_coef_p, contr_coef_d, coords, basis, pairs,
                                 shell_xyz);
    if (rc) return rc;
    const size_t npairs = (size_t)pairs.class_off[NPC], nprim = pairs.P.size();
    // layout inside the array: tables | shells | pairs | primitive pairs | results
    size_t off = 0;
    const size_t o_tab = off;
    off = align256(off + (size_t)RYS_TABLE_SIZE * sizeof(double));
    const size_t o_xyz = off;
    off = align256(off + (size_t)nsh * sizeof(double4));
    const size_t o_bf0 = off;
    off = align256(off + (size_t)nsh * sizeof(int));
    const size_t o_psh = off;
    off = align256(off + npairs * sizeof(int2));
    const size_t o_p0 = off;
    off = align256(off + npairs * sizeof(int));
    const size_t o_np = off;
    off = align256(off + npairs * sizeof(int));
    const size_t o_P = off;
    off = align256(off + nprim * sizeof(double4));
    const size_t o_X = off;
    off = align256(off + nprim * sizeof(double2));
    const size_t o_out = off;
    off = align256(off + npairs * sizeof(double));
    if (off > NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "liberi_schwarz_noalloc: basis needs %zu bytes of device scratch, limit is %zu (%zu pairs, %zu "
                 "primitive pairs); use liberi_c_schwarz",
                 off, NOALLOC_SCRATCH_BYTES, npairs, nprim);
        return set_error(LIBERI_E_NOMEM, msg);
    }
    std::lock_guard<std::mutex> lock(g_mu);
    unsigned char *base = nullptr;
    rc = setup_device(&base);
    if (rc) return rc;
    (void)o_tab;
    cudaError_t e = cudaSuccess;
    std::vector<int> bf0(nsh);
    for (int s = 0; s < nsh; s++) bf0[s] = basis.atom_loc[s] - 1;
    struct Part {
        size_t off;
        const void *src;
        size_t bytes;
    } parts[] = {{o_xyz, shell_xyz.data(), (size_t)nsh * sizeof(double4)},
                 {o_bf0, bf0.data(), (size_t)nsh * sizeof(int)},
                 {o_psh, pairs.shell.data(), npairs * sizeof(int2)},
                 {o_p0, pairs.prim0.data(), npairs * sizeof(int)},
                 {o_np, pairs.nprim.data(), npairs * sizeof(int)},
                 {o_P, pairs.P.data(), nprim * sizeof(double4)},
                 {o_X, pairs.X.data(), nprim * sizeof(double2)}};
    for (const Part &pt : parts) {
        if (pt.bytes == 0) continue;
        e = cudaMemcpy(base + pt.off, pt.src, pt.bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess)
            return set_error(LIBERI_E_DEVICE, (std::string("liberi_schwarz_noalloc: upload failed: ") +
                                               cudaGetErrorString(e)).c_str());
    }
    double *d_out = (double *)(base + o_out);
    e = cudaMemset(d_out, 0, npairs * sizeof(double));
    DevBasis db;
    db.shell_xyz = (const double4 *)(base + o_xyz);
    db.shell_bf0 = (const int *)(base + o_bf0);
    db.pair_shell = (const int2 *)(base + o_psh);
    db.pair_prim0 = (const int *)(base + o_p0);
    db.pair_nprim = (const int *)(base + o_np);
    db.prim_P = (const double4 *)(base + o_P);
    db.prim_X = (const double2 *)(base + o_X);
    db.prim_PAf = nullptr;  // the Schwarz kernels are FP64 only
    db.prim_bound = nullptr;
    const double *tab = (const double *)(base + o_tab);
    for (int c = 0; c < NPC && e == cudaSuccess; c++) {
        const int o = pairs.class_off[c], n = pairs.class_off[c + 1] - o;
        e = launch_schwarz(c, n, o, db, tab, d_out + o, 0);
    }
    std::vector<double> per_pair(npairs);
    if (e == cudaSuccess && npairs > 0)
        e = cudaMemcpy(per_pair.data(), d_out, npairs * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return set_error(LIBERI_E_DEVICE, (std::string("liberi_schwarz_noalloc: ") + cudaGetErrorString(e)).c_str());
    const size_t ntri = (size_t)nsh * (nsh + 1) / 2;
    std::fill(schwrz_out, schwrz_out + ntri, 0.0);
    for (size_t p = 0; p < npairs; p++) {
        const int hi = std::max(pairs.ish[p], pairs.jsh[p]) + 1, lo = std::min(pairs.ish[p], pairs.jsh[p]) + 1;
        schwrz_out[(size_t)hi * (hi - 1) / 2 + lo - 1] = per_pair[p];
    }
    return LIBERI_OK;
}
