/*
 * liberi_b200.h -- C ABI of the B200 RHF Fock-build engine.
 *
 * Drop-in for libERI's handle API and its GAMESS direct-link wrapper.  Every
 * entry point returns an int status: 0 on success, a negative LIBERI_E_* code
 * otherwise; liberi_c_last_error() returns the message of the calling thread's
 * last failure.  The reference aborts with `error stop 1` instead; the Fortran
 * shim (gms_liberi_b200/fortran/liberi_b200_interface.F90) maps a non-zero
 * status back to `error stop 1`.
 *
 * Layout conventions follow the reference exactly:
 *   - density and Fock matrices are packed lower triangles of length
 *     n(n+1)/2, element (i,j), i>=j, 1-based, at ia(i)+j with ia(i)=i(i-1)/2
 *     (src/liberi_shell_pair.F90:131-133, src/rhf/rot_axis/int0000.F90:273-283);
 *   - schwrz_int is packed the same way over shells;
 *   - sh_loc, atom_num, atom_loc are 1-based; ang_mom 1=s 2=p 3=d 4=f;
 *     Cartesian d order xx,yy,zz,xy,xz,yz with sqrt(3) on xy,xz,yz; f order
 *     xxx,yyy,zzz,xxy,xxz,xyy,yyz,xzz,yzz,xyz with sqrt(5) on the six mixed
 *     components and sqrt(15) on xyz (src/rhf/rys/int3011_rysgen.F90).
 * All integer arguments are int32_t (the reference requires c_int at the
 * boundary), all real arrays double.
 */
#ifndef LIBERI_B200_H
#define LIBERI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct liberi_handle_s *liberi_handle;

enum {
    LIBERI_OK = 0,
    LIBERI_E_ARG = -1,        /* bad pointer, size or option */
    LIBERI_E_STATE = -2,      /* call before setup, after cleanup, ... */
    LIBERI_E_SIZE = -3,       /* matrix_size != num_bas(num_bas+1)/2 */
    LIBERI_E_DEVICE = -4,     /* CUDA error */
    LIBERI_E_NOMEM = -5,      /* device allocation failed or over limit */
    LIBERI_E_UNSUPPORTED = -6 /* num_bas > 65535; f shells in the Schwarz generator or a batch; NCCL absent */
};

/* ---- handle API: src/interface/liberi_interface.F90 --------------------- */

/* liberi_create(handle)                      liberi_interface.F90:46-55 */
int liberi_c_create(liberi_handle *handle);

/* liberi_destroy(handle): cleans up if still initialised.       :57-70 */
int liberi_c_destroy(liberi_handle handle);

/* liberi_setup(handle, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num,
 * sh_loc, atom_num, atom_loc, start_bas, end_bas, exponents, contr_coef_s,
 * contr_coef_p, contr_coef_d, contr_coef_f, coords, schwrz_int, my_rank,
 * num_procs).  Deep-copies every input, builds shell pairs and the screened
 * quartet plan on the device.  Calling it on an initialised handle cleans up
 * first.                                                          :72-200 */
int liberi_c_setup(liberi_handle handle, int32_t nsh, int32_t natoms, int32_t num_bas,
                   int32_t mxgtot, const int32_t *ang_mom, const int32_t *contr_num,
                   const int32_t *sh_loc, const int32_t *atom_num, const int32_t *atom_loc,
                   const int32_t *start_bas, const int32_t *end_bas, const double *exponents,
                   const double *contr_coef_s, const double *contr_coef_p,
                   const double *contr_coef_d, const double *contr_coef_f, const double *coords,
                   const double *schwrz_int, int32_t my_rank, int32_t num_procs);

/* liberi_fock_build(handle, density, fock, matrix_size): overwrites fock
 * with this rank's partial two-electron Fock contribution (host buffers).
 * The caller reduces partials across ranks, as GAMESS does with DDI_GSUMF.
 *                                                                 :202-227 */
int liberi_c_fock_build(liberi_handle handle, const double *density, double *fock,
                        int32_t matrix_size);

/* liberi_cleanup(handle): frees device state; no-op if not set up. :229-260 */
int liberi_c_cleanup(liberi_handle handle);

/* ---- GAMESS direct-link wrapper: src/interface/gms_liberi_wrapper.F90 ---- */

/* liberi_init(natoms, num_bas, nsh, mxgtot, ...): note natoms first.  :29-100 */
int liberi_c_init(int32_t natoms, int32_t num_bas, int32_t nsh, int32_t mxgtot,
                  const int32_t *ang_mom, const int32_t *contr_num, const int32_t *sh_loc,
                  const int32_t *atom_num, const int32_t *atom_loc, const int32_t *start_bas,
                  const int32_t *end_bas, const double *exponents, const double *contr_coef_s,
                  const double *contr_coef_p, const double *contr_coef_d,
                  const double *contr_coef_f, const double *coords, const double *schwrz_int,
                  int32_t my_rank, int32_t num_procs);
/* liberi_fock(density, fock, n) with the wrapper's size check.    :103-131 */
int liberi_c_fock(const double *density, double *fock, int32_t n);
/* liberi_finalize()                                               :134-146 */
int liberi_c_finalize(void);

/* ---- extensions without a reference counterpart ------------------------- */

/* Message of the calling thread's last failure (NUL-terminated, truncated). */
int liberi_c_last_error(char *buf, int32_t len);

/* Runtime options; defaults reproduce the reference's compile-time constants.
 *   "schwarz_cut"  (5e-11, cutoff_schwarz, src/liberi_parameters.F90:38)
 *   "eri_cut"      (5e-11, the digestion literal, e.g. int0002.F90:403)
 *   "fp32_cut"     (1e-7; quartets with xint_ab*xint_cd*max|D| below it run
 *                   in FP32 when "precision" is 1)
 *   "fp32_prim"    (1e-8; inside those FP32 quartets, a primitive quartet
 *                   whose Schwarz bound b_ab*b_cd*max|D| is below
 *                   fp32_prim*fp32_cut is skipped: each skipped contribution
 *                   to F is below 1e-8 of the cut, about the tier's own
 *                   rounding error; 0 keeps every primitive; FP64 quartets
 *                   never skip primitives)
 *   "precision"    (0 = all FP64, 1 = mixed FP32/FP64)
 *   "device"       (CUDA device ordinal used by the next setup, default 0)
 *   "class_mask"   (bit k set = run class k of the driver order; default all 21)
 *   "rank_split"   (0 = the reference's per-kernel split of quartets over
 *                   my_rank/num_procs, reproducing its partial F per rank;
 *                   1 = cost-balanced contiguous slices of every class's work,
 *                   the same total F with even per-rank time; before setup)
 *   "tile_mask"    (bit k set = class k may stage rows of F in a shared-memory
 *                   tile, where it fits; default none: F is updated with FP64
 *                   atomics in L2, faster on B200 for every class measured)
 *   "overlap"      (1 = streams forked from and joined back into the
 *                   build's stream: builds of at most 25 million screened
 *                   quartets spread their classes over 8 streams (while "fan"
 *                   is 1); larger ones run every class's FP64 task list beside
 *                   the FP32 lists (mixed precision) or the classes of
 *                   "side_mask" beside the others (FP64) on a second stream;
 *                   default 1; off while "timing")
 *   "side_mask"    (bit k set = FP64 builds launch class k on the second
 *                   stream; default the high-L and low-occupancy classes
 *                   measured faster there on C60)
 *   "fan"          (1 = the 8-stream spread of small builds above, default 1;
 *                   set 0 where many handles build at once and already fill
 *                   the GPU, as the serving loop does)
 *   "timing"       (1 = record per-class device times for liberi_c_get_stats)
 *   "max_device_bytes" (0 = no limit; otherwise liberi_c_setup fails with
 *                   LIBERI_E_NOMEM, before any device work, when the basis
 *                   and plans would need more device bytes than this)
 * Options set before liberi_c_setup apply to it; cut options may also be
 * changed between builds (the quartet plan is rebuilt on the next build). */
int liberi_c_set_option(liberi_handle handle, const char *name, double value);
int liberi_c_get_option(liberi_handle handle, const char *name, double *value);

/* Fock build on device-resident packed buffers (no host copies), enqueued on
 * `stream` (a cudaStream_t, NULL = the handle's own stream); does not
 * synchronise.  Used for device-resident benchmarking and graph capture.
 * Builds of one handle share its device scratch (the full copy of D the
 * kernels read, the mixed-precision task lists): enqueue them on one stream
 * (or order them), as a handle is not thread-safe in the reference. */
int liberi_c_fock_build_device(liberi_handle handle, const double *d_density, double *d_fock,
                               void *stream);

/* Open-shell (UHF) Fock build.  No counterpart in the reference: its MDI
 * plugin registers ">AO_DENS_B" and "<FOCK_B" (liberi_mdi_api.F90:395-421)
 * but libERI builds closed-shell F only.  With the alpha and beta densities
 * (packed like D) it returns, this rank's partials in the units of
 * liberi_c_fock_build,
 *     F_alpha = J(D_alpha + D_beta) - K(2 D_alpha),
 *     F_beta  = J(D_alpha + D_beta) - K(2 D_beta),
 * where J and K are the Coulomb and exchange updates of DIRFCK
 * (int0000.F90:241-311), so that D_alpha = D_beta = D/2 gives the RHF F.
 * Two builds over the same screened quartets; mixed precision splits at the
 * largest element of both densities.  The host variant keeps D_alpha/F_alpha
 * in the handle's buffers and the beta pair in a scratch allocation. */
int liberi_c_fock_build_uhf(liberi_handle handle, const double *density_a, const double *density_b,
                            double *fock_a, double *fock_b, int32_t matrix_size);
int liberi_c_fock_build_uhf_device(liberi_handle handle, const double *d_density_a, const double *d_density_b,
                                   double *d_fock_a, double *d_fock_b, void *stream);

/* Schwarz table generator: schwrz_out[ia(max)+min] = sqrt(max_components
 * |(ab|ab)|) over shell pairs, computed on the device (GAMESS supplies this
 * table to the reference, liberi_interface.F90:128-129).  s/p/d/f shells;
 * contr_coef_f may be NULL for bases without f shells. */
int liberi_c_schwarz(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot,
                     const int32_t *ang_mom, const int32_t *contr_num, const int32_t *sh_loc,
                     const int32_t *atom_num, const int32_t *atom_loc, const double *exponents,
                     const double *contr_coef_s, const double *contr_coef_p, const double *contr_coef_d,
                     const double *contr_coef_f, const double *coords, double *schwrz_out);

/* Schwarz table without device allocation.  No counterpart in the reference:
 * the inputs and output of liberi_c_schwarz for s/p/d bases (no f
 * coefficients; f shells are rejected), for callers that cannot call
 * cudaMalloc (their device memory is already committed to their own pool, or
 * their allocation policy forbids ad-hoc cudaMalloc/cudaFree).  Its device
 * scratch is one static array of LIBERI_NOALLOC_SCRATCH_BYTES that every GPU
 * it has run on holds until exit.  CUDA loads device code lazily, so the
 * array is committed by the first call on each device (LIBERI_E_NOMEM if that
 * fails): make that call at start-up, before a pool claims the memory, and
 * before any stream capture.  Bases that need more scratch are rejected with
 * LIBERI_E_NOMEM before any GPU work.  Calls are serialised and share the
 * array; uses that overlap on the GPU would race. */
#define LIBERI_NOALLOC_SCRATCH_BYTES (8u << 20)
int liberi_c_schwarz_noalloc(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot,
                             const int32_t *ang_mom, const int32_t *contr_num, const int32_t *sh_loc,
                             const int32_t *atom_num, const int32_t *atom_loc, const double *exponents,
                             const double *contr_coef_s, const double *contr_coef_p,
                             const double *contr_coef_d, const double *coords, double *schwrz_out);

/* Per-kernel statistics of the last build, the 21 s/p/d rows in the reference
 * driver order (liberi_driver.F90:69-102; the f classes through
 * liberi_c_get_class_stats):
 *   quartets[k]     screened shell quartets owned by this rank
 *   fp32_quartets[k] of those, evaluated in FP32
 *   prim_quartets[k] primitive quartets (after mu*R^2 > 50 pair removal)
 *   kernel_ms[k]    device time of the class (0 unless timing is enabled)  */
typedef struct {
    int64_t quartets[21];
    int64_t fp32_quartets[21];
    int64_t prim_quartets[21];
    double kernel_ms[21];
    double build_ms;
    int64_t device_bytes;
} liberi_stats;
int liberi_c_get_stats(liberi_handle handle, liberi_stats *stats);
/* Class k of all 55 (0..20 the s/p/d kernels, 21..54 the f block in the
 * driver's order, liberi_driver.F90:103-160): out[0] screened shell quartets
 * owned by this rank, out[1] primitive quartets.  No counterpart in the
 * reference. */
int liberi_c_get_class_stats(liberi_handle handle, int32_t k, int64_t *out);

/* Fingerprint of the screened-quartet set, for parity checks.  No counterpart
 * in the reference (its kernels enumerate the set implicitly: pre-screen and
 * product test, e.g. int0001.F90:67-121; no product test in
 * int2222_rysgen.F90:428-436).  For each class in driver order, out[3k+0..2]
 * = {number of quartets, sum, xor} of a 64-bit hash of every quartet that the
 * class kernels evaluate for this rank over the task lists of the last build
 * (the static plan for an FP64 build or before any build; the per-build FP64
 * and FP32 lists of a mixed-precision build).  The hash of a quartet depends
 * only on its four shells (0-based), not on pair orientation or bra/ket
 * order: unordered shell pairs s1<<16|s2 (s1 >= s2), the larger pair key
 * <<32 | the smaller, mixed by the 64-bit finaliser x ^= x>>33,
 * x *= 0xff51afd7ed558ccd, x ^= x>>33, x *= 0xc4ceb9fe1a85ec53, x ^= x>>33.
 * Runs on the device, synchronous; fails if options changed since the last
 * build (the plan would be rebuilt first). */
int liberi_c_quartet_fingerprint(liberi_handle handle, uint64_t *out);
/* The same for all 55 classes (out[3*55]; the f classes always evaluate their
 * static FP64 lists). */
int liberi_c_quartet_fingerprint_all(liberi_handle handle, uint64_t *out);

/* Device bytes liberi_c_setup would allocate for this basis at this Schwarz
 * cut (host-only dry run of the pair and plan construction, no device
 * access): the admission figure of a serving loop.  No counterpart in the
 * reference. */
int liberi_c_setup_bytes(int32_t nsh, int32_t natoms, int32_t num_bas, int32_t mxgtot, const int32_t *ang_mom,
                         const int32_t *contr_num, const int32_t *sh_loc, const int32_t *atom_num,
                         const int32_t *atom_loc, const double *exponents, const double *contr_coef_s,
                         const double *contr_coef_p, const double *contr_coef_d, const double *contr_coef_f,
                         const double *coords, const double *schwrz_int, double schwarz_cut, int64_t *bytes);

/* Batched Fock builds over several set-up handles (one molecule each): one
 * launch per quartet class covers every molecule (a persistent multi-molecule
 * work list), preceded by one launch that zeroes every F.  No counterpart in
 * the reference.  Handles must have s/p/d bases (f shells: LIBERI_E_UNSUPPORTED)
 * and share device, cuts and precision (FP64, or
 * mixed with one fp32_cut: each iteration then splits every molecule's work
 * at its own max|D| on the device, inside the captured graph) and use one rank.
 *   bind:     device density / Fock buffer of every molecule (kept by address);
 *   fock_build: enqueue one SCF iteration of all molecules on `stream` (NULL:
 *             the batch's own stream);
 *   capture / launch: record that iteration once as a CUDA graph and replay it;
 *   autotune: time each class at 128..2048 kets per CTA task, keep the
 *             fastest (chunks_out[21] may be NULL), re-capture if captured.
 * The batch reads each handle's plans as they are at create: changing a
 * handle's options, setting it up again or cleaning it up afterwards needs a
 * new batch.  Destroy the batch before its handles. */
typedef struct liberi_batch_s *liberi_batch;
int liberi_c_batch_create(liberi_batch *batch, const liberi_handle *handles, int32_t n);
int liberi_c_batch_bind(liberi_batch batch, const double *const *d_density, double *const *d_fock);
int liberi_c_batch_fock_build(liberi_batch batch, void *stream);
int liberi_c_batch_capture(liberi_batch batch);
int liberi_c_batch_launch(liberi_batch batch, void *stream);
int liberi_c_batch_synchronize(liberi_batch batch);
int liberi_c_batch_autotune(liberi_batch batch, int32_t reps, int32_t *chunks_out);
int liberi_c_batch_destroy(liberi_batch batch);

/* Autotuner for one handle: per class, the fastest kernel shape variant
 * (A components per pass and resident CTAs per SM, 0..2) and number of kets
 * per CTA task (128..2048) on the handle's own device buffers (their
 * contents are overwritten), and for a mixed-precision handle the fastest
 * FP32-tier shape; the plan is rebuilt with the choice.  No counterpart in
 * the reference. */
int liberi_c_autotune(liberi_handle handle, int32_t reps, int32_t *chunks_out);
/* Kernel shape variant of class k (driver order 0..20) for precision 0
 * (FP64) or 1 (FP32 tier); variant 0 is the default, a variant that is not
 * distinct for a class runs variant 0.  No counterpart in the reference. */
int liberi_c_set_class_variant(liberi_handle handle, int32_t k, int32_t precision, int32_t variant);
int liberi_c_get_class_variant(liberi_handle handle, int32_t k, int32_t precision, int32_t *variant);

/* Rys roots u_i = t_i^2 and weights w_i (sum w_i = F_0(T)) for n = 1..5 from
 * the engine's piecewise tables, evaluated on the host exactly as the device
 * does; the large-T limit is used for T > thr (strict) or T >= thr. */
int liberi_c_rys_eval(int32_t n, double T, double thr, int32_t strict, double *u, double *w);
/* The FP32 tier's tables (intervals of width 1/8, degree 3), evaluated in
 * single precision exactly as the device does.  No counterpart in the
 * reference. */
int liberi_c_rys_eval_f32(int32_t n, float T, float thr, int32_t strict, float *u, float *w);
/* The f classes' tables (n = 1..7 roots on [0, 65)), evaluated as the f
 * kernel does.  No counterpart in the reference. */
int liberi_c_rys7_eval(int32_t n, double T, double thr, int32_t strict, double *u, double *w);

/* Device microbenchmarks on the current device (roofline denominators):
 *   kind 0: FP64 FMA throughput, TFLOP/s
 *   kind 1: FP32 FMA throughput, TFLOP/s
 *   kind 2: FP64 atomicAdd throughput into a 405,450-element (3.2 MB,
 *           L2-resident) array at random addresses, Gatomic/s
 *   kind 3: shared-memory FP64 atomicAdd throughput (3,600-element block
 *           array, random addresses), Gatomic/s */
int liberi_c_microbench(int32_t kind, double *result);

/* Name of kernel class k (0..54: the 21 s/p/d classes, then the f block),
 * e.g. "int2222"; NULL if out of range. */
const char *liberi_c_kernel_name(int32_t k);

/* ---- MDI plugin command set (liberi_mdi_api.F90:194-428), transport-free ----
 * The reference's plugin answers MDI commands from GAMESS: '>' commands
 * deliver data (accumulated in a persistent state), '>SCHWZ_INT' runs
 * liberi_setup, '>AO_DENS' delivers D, '<FOCK' returns F.  This object is that
 * state machine; an MDI plugin shim (MDI_Plugin_init_ERI / open / close,
 * linked against the MDI library) receives each command, asks
 * liberi_c_mdi_payload for the element type and count it carries, moves the
 * payload with MDI_Recv / MDI_Send and calls liberi_c_mdi_execute.  '<FOCK'
 * writes this rank's partial F; the shim sums the ranks' partials (MPI_Reduce
 * in the reference, an NCCL reduction on GPUs) before sending.  'EXIT' sets
 * *terminate and keeps the state for the next launch; 'EXIT_CONVERGED' also
 * releases the handle.  Open shell: after '>AO_DENS_B' (the beta density),
 * '<FOCK' returns the alpha F of liberi_c_fock_build_uhf and '<FOCK_B' the
 * beta F of the same build (LIBERI_E_STATE without one); commands the
 * reference registers without handling ('<COORDS', '>FOCK', '>FOCK_B') and
 * unknown ones return LIBERI_E_ARG.
 * '>RANK_ID' / '>NUM_PROCS' (registered, not handled by the reference) set the
 * rank split used at setup; liberi_c_mdi_create takes the same from the
 * shim's communicator. */
typedef struct liberi_mdi_s *liberi_mdi;
typedef struct liberi_comm_s *liberi_comm;
enum { LIBERI_MDI_NONE = 0, LIBERI_MDI_INT = 1, LIBERI_MDI_DOUBLE = 2, LIBERI_MDI_CHAR = 3 };
int liberi_c_mdi_create(liberi_mdi *state, int32_t my_rank, int32_t num_procs);
int liberi_c_mdi_payload(liberi_mdi state, const char *command, int32_t *type, int64_t *count);
int liberi_c_mdi_execute(liberi_mdi state, const char *command, void *buffer, int64_t count, int32_t *terminate);
int liberi_c_mdi_destroy(liberi_mdi state);
/* Sum the ranks' partial F over an NCCL communicator inside '<FOCK' (and
 * '<FOCK_B'): every rank's buffer then holds the total, which the shim sends
 * from rank 0 without its own MPI_Reduce.  NULL restores the partial. */
int liberi_c_mdi_set_comm(liberi_mdi state, liberi_comm comm);

/* ---- the sum of the ranks' partial Fock matrices over NCCL ----------------
 * libERI leaves the sum to its caller (MPI_Reduce in the MDI plugin,
 * liberi_mdi_api.F90:411-414).  Here it runs on the devices: rank 0 makes a
 * unique id (LIBERI_COMM_ID_BYTES bytes), the caller broadcasts it (MPI_Bcast
 * in the shim), every rank creates its communicator on its device (this call
 * waits for all ranks), and liberi_c_comm_allreduce sums packed F in device
 * memory (NVLink / NVSwitch) on `stream` (NULL: the communicator's own).
 * liberi_c_comm_reduce_host sums host buffers through a device copy.
 * NCCL (libnccl.so.2) is loaded on first use; without it these calls return
 * LIBERI_E_UNSUPPORTED.  No counterpart in the reference. */
#define LIBERI_COMM_ID_BYTES 128
int liberi_c_comm_unique_id(uint8_t *id_out);
int liberi_c_comm_create(liberi_comm *comm, const uint8_t *id, int32_t rank, int32_t nranks, int32_t device);
int liberi_c_comm_allreduce(liberi_comm comm, const double *d_send, double *d_recv, int64_t count, void *stream);
int liberi_c_comm_reduce_host(liberi_comm comm, const double *in, double *out, int64_t count);
int liberi_c_comm_destroy(liberi_comm comm);

#ifdef __cplusplus
}
#endif
#endif
