// comm.cpp -- sum of the ranks' partial Fock matrices over NCCL.
//
// libERI returns each rank's partial F and leaves the sum to its caller: the
// MDI plugin reduces with MPI_Reduce before '<FOCK' is sent
// (src/interface/liberi_mdi_api.F90:411-414), GAMESS's direct link with
// DDI_GSUMF.  On GPUs the partials already live in device memory, so the sum
// runs there: an NCCL communicator over the ranks' devices (NVLink / NVSwitch,
// in-switch reduction where NCCL uses it) and one all-reduce of the packed F.
// The caller creates the communicator from a unique id that rank 0 makes and
// broadcasts (the MDI shim does it with MPI_Bcast).  NCCL is loaded on first
// use (dlopen "libnccl.so.2": the process's copy if one is loaded already),
// so the library itself loads where NCCL is absent.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "../../include/liberi_b200.h"
#include "engine.h"

namespace {

struct NcclApi {
    bool ok = false;
    std::string err;
    ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char *(*error_string)(ncclResult_t) = nullptr;
};
NcclApi g_nccl;
std::once_flag g_nccl_once;

const NcclApi &nccl() {
    std::call_once(g_nccl_once, [] {
        void *lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!lib) {
            g_nccl.err = std::string("cannot load libnccl.so.2: ") + dlerror();
            return;
        }
        g_nccl.get_unique_id = (decltype(g_nccl.get_unique_id))dlsym(lib, "ncclGetUniqueId");
        g_nccl.comm_init_rank = (decltype(g_nccl.comm_init_rank))dlsym(lib, "ncclCommInitRank");
        g_nccl.all_reduce = (decltype(g_nccl.all_reduce))dlsym(lib, "ncclAllReduce");
        g_nccl.comm_destroy = (decltype(g_nccl.comm_destroy))dlsym(lib, "ncclCommDestroy");
        g_nccl.error_string = (decltype(g_nccl.error_string))dlsym(lib, "ncclGetErrorString");
        g_nccl.ok = g_nccl.get_unique_id && g_nccl.comm_init_rank && g_nccl.all_reduce && g_nccl.comm_destroy &&
                    g_nccl.error_string;
        if (!g_nccl.ok) g_nccl.err = "libnccl.so.2 lacks an expected entry point";
    });
    return g_nccl;
}

int nccl_fail(const char *what, ncclResult_t r) {
    char msg[256];
    snprintf(msg, sizeof msg, "%s: %s", what, nccl().error_string ? nccl().error_string(r) : "NCCL error");
    return liberi::set_error(LIBERI_E_DEVICE, msg);
}

}  // namespace

struct liberi_comm_s {
    ncclComm_t comm = nullptr;
    int device = 0, rank = 0, nranks = 1;
    cudaStream_t stream = nullptr;
    double *scratch = nullptr;  // device staging of host buffers (liberi_c_comm_reduce_host)
    size_t scratch_n = 0;
};

namespace liberi {
int comm_device(liberi_comm c) { return c ? c->device : -1; }
}  // namespace liberi

extern "C" {

int liberi_c_comm_unique_id(uint8_t *id_out) {
    if (!id_out) return liberi::set_error(LIBERI_E_ARG, "liberi_comm_unique_id: null output");
    const NcclApi &api = nccl();
    if (!api.ok) return liberi::set_error(LIBERI_E_UNSUPPORTED, api.err.c_str());
    ncclUniqueId id;
    ncclResult_t r = api.get_unique_id(&id);
    if (r != ncclSuccess) return nccl_fail("ncclGetUniqueId", r);
    std::memcpy(id_out, id.internal, LIBERI_COMM_ID_BYTES);
    return LIBERI_OK;
}

int liberi_c_comm_create(liberi_comm *out, const uint8_t *id, int32_t rank, int32_t nranks, int32_t device) {
    if (!out || !id || nranks < 1 || rank < 0 || rank >= nranks)
        return liberi::set_error(LIBERI_E_ARG, "liberi_comm_create: bad arguments");
    const NcclApi &api = nccl();
    if (!api.ok) return liberi::set_error(LIBERI_E_UNSUPPORTED, api.err.c_str());
    if (device < 0) {  // one rank per visible device, in rank order
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
            return liberi::set_error(LIBERI_E_DEVICE, "liberi_comm_create: no CUDA device");
        device = rank % ndev;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return liberi::set_error(LIBERI_E_DEVICE, "liberi_comm_create: bad device");
    liberi_comm c = new (std::nothrow) liberi_comm_s();
    if (!c) return liberi::set_error(LIBERI_E_NOMEM, "liberi_comm_create: out of host memory");
    c->device = device;
    c->rank = rank;
    c->nranks = nranks;
    ncclUniqueId uid;
    std::memcpy(uid.internal, id, LIBERI_COMM_ID_BYTES);
    int rc = LIBERI_OK;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = liberi::set_error(LIBERI_E_DEVICE, "liberi_comm_create: stream");
    if (!rc) {
        ncclResult_t r = api.comm_init_rank(&c->comm, nranks, uid, rank);  // waits for every rank
        if (r != ncclSuccess) rc = nccl_fail("ncclCommInitRank", r);
    }
    if (prev >= 0) cudaSetDevice(prev);
    if (rc) {
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return rc;
    }
    *out = c;
    return LIBERI_OK;
}

int liberi_c_comm_allreduce(liberi_comm c, const double *d_send, double *d_recv, int64_t count, void *stream) {
    if (!c || !d_send || !d_recv || count < 0) return liberi::set_error(LIBERI_E_ARG, "liberi_comm_allreduce: bad arguments");
    if (count == 0) return LIBERI_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    ncclResult_t r = nccl().all_reduce(d_send, d_recv, (size_t)count, ncclFloat64, ncclSum, c->comm,
                                       stream ? (cudaStream_t)stream : c->stream);
    if (prev >= 0) cudaSetDevice(prev);
    if (r != ncclSuccess) return nccl_fail("ncclAllReduce", r);
    return LIBERI_OK;
}

int liberi_c_comm_reduce_host(liberi_comm c, const double *in, double *out, int64_t count) {
    if (!c || !in || !out || count < 0) return liberi::set_error(LIBERI_E_ARG, "liberi_comm_reduce_host: bad arguments");
    if (count == 0) return LIBERI_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    cudaError_t e = cudaSuccess;
    if (c->scratch_n < (size_t)count) {
        if (c->scratch) cudaFree(c->scratch);
        c->scratch = nullptr;
        c->scratch_n = 0;
        e = cudaMalloc((void **)&c->scratch, (size_t)count * sizeof(double));
        if (e == cudaSuccess) c->scratch_n = (size_t)count;
    }
    const size_t bytes = (size_t)count * sizeof(double);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->scratch, in, bytes, cudaMemcpyHostToDevice, c->stream);
    int rc = LIBERI_OK;
    if (e == cudaSuccess) rc = liberi_c_comm_allreduce(c, c->scratch, c->scratch, count, c->stream);
    if (e == cudaSuccess && !rc) e = cudaMemcpyAsync(out, c->scratch, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && !rc) e = cudaStreamSynchronize(c->stream);
    if (prev >= 0) cudaSetDevice(prev);
    if (rc) return rc;
    if (e != cudaSuccess) return liberi::set_error(LIBERI_E_DEVICE, cudaGetErrorString(e));
    return LIBERI_OK;
}

int liberi_c_comm_destroy(liberi_comm c) {
    if (!c) return liberi::set_error(LIBERI_E_ARG, "liberi_comm_destroy: null communicator");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    if (c->comm) nccl().comm_destroy(c->comm);
    if (c->scratch) cudaFree(c->scratch);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (prev >= 0) cudaSetDevice(prev);
    delete c;
    return LIBERI_OK;
}

}  // extern "C"
