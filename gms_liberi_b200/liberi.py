"""Python front end of the B200 Fock-build engine (ctypes over the C ABI in
include/liberi_b200.h).

Mirrors libERI's Fortran API for this path:

* handle API (src/interface/liberi_interface.F90): ``liberi_create``,
  ``liberi_setup``, ``liberi_fock_build``, ``liberi_cleanup``,
  ``liberi_destroy`` with the reference's argument lists and meanings;
* GAMESS direct-link wrapper (src/interface/gms_liberi_wrapper.F90):
  ``liberi_init`` (natoms first), ``liberi_fock``, ``liberi_finalize``.

Where the reference stops with ``error stop 1`` these raise ``LiberiError``
carrying the C status code and message.  There is no CPU fallback: importing
this module fails if the CUDA library has not been built.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libliberi_b200.so")

KERNELS = ["int0000", "int0001", "int0011", "int0111", "int0101", "int1111",
           "int0002", "int0012", "int0102", "int0112", "int0022", "int0122",
           "int1102", "int0202", "int2211", "int2121", "int2120", "int2111",
           "int2220", "int2221", "int2222"]
# the f block of the reference driver, in its order (src/liberi_driver.F90:103-160)
KERNELS_F = ["int3333", "int0030", "int0031", "int0032", "int1030", "int3330", "int3011", "int3020",
             "int2130", "int2230", "int3030", "int3110", "int3111", "int3120", "int3121", "int2231",
             "int3130", "int3131", "int3210", "int3331", "int3211", "int3220", "int3221", "int3222",
             "int3230", "int3231", "int3232", "int3300", "int3310", "int3311", "int3320", "int3321",
             "int3322", "int3332"]
KERNELS_ALL = KERNELS + KERNELS_F
NCLASS = len(KERNELS_ALL)

EXPORTS = ["liberi_c_create", "liberi_c_destroy", "liberi_c_setup", "liberi_c_fock_build",
           "liberi_c_cleanup", "liberi_c_init", "liberi_c_fock", "liberi_c_finalize",
           "liberi_c_last_error", "liberi_c_set_option", "liberi_c_get_option",
           "liberi_c_fock_build_device", "liberi_c_schwarz", "liberi_c_get_stats",
           "liberi_c_kernel_name", "liberi_c_rys_eval", "liberi_c_microbench",
           "liberi_c_schwarz_noalloc", "liberi_c_batch_create", "liberi_c_batch_bind",
           "liberi_c_batch_fock_build", "liberi_c_batch_capture", "liberi_c_batch_launch",
           "liberi_c_batch_synchronize", "liberi_c_batch_autotune", "liberi_c_batch_destroy",
           "liberi_c_autotune", "liberi_c_rys_eval_f32", "liberi_c_setup_bytes",
           "liberi_c_set_class_variant", "liberi_c_get_class_variant", "liberi_c_mdi_create",
           "liberi_c_mdi_payload", "liberi_c_mdi_execute", "liberi_c_mdi_destroy",
           "liberi_c_quartet_fingerprint", "liberi_c_fock_build_uhf", "liberi_c_fock_build_uhf_device",
           "liberi_c_mdi_set_comm", "liberi_c_comm_unique_id", "liberi_c_comm_create", "liberi_c_comm_allreduce",
           "liberi_c_comm_reduce_host", "liberi_c_comm_destroy", "liberi_c_get_class_stats",
           "liberi_c_quartet_fingerprint_all", "liberi_c_rys7_eval"]

_I32P = ctypes.POINTER(ctypes.c_int32)
_F64P = ctypes.POINTER(ctypes.c_double)


class LiberiError(RuntimeError):
    """A failed C-ABI call; ``code`` is the negative LIBERI_E_* status."""

    def __init__(self, code, msg):
        super().__init__("liberi error %d: %s" % (code, msg))
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [("quartets", ctypes.c_int64 * 21), ("fp32_quartets", ctypes.c_int64 * 21),
                ("prim_quartets", ctypes.c_int64 * 21), ("kernel_ms", ctypes.c_double * 21),
                ("build_ms", ctypes.c_double), ("device_bytes", ctypes.c_int64)]


_lib = None


def lib():
    """Load the CUDA library; raises if it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libliberi_b200.so not built at %s; run __graft_entry__.build()" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        H = ctypes.c_void_p
        L.liberi_c_create.argtypes = [ctypes.POINTER(H)]
        L.liberi_c_destroy.argtypes = [H]
        L.liberi_c_cleanup.argtypes = [H]
        L.liberi_c_setup.argtypes = [H, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                     _I32P, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P,
                                     _F64P, _F64P, _F64P, _F64P, _F64P, _F64P, _F64P,
                                     ctypes.c_int32, ctypes.c_int32]
        L.liberi_c_fock_build.argtypes = [H, _F64P, _F64P, ctypes.c_int32]
        L.liberi_c_fock_build_device.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.liberi_c_init.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    _I32P, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P,
                                    _F64P, _F64P, _F64P, _F64P, _F64P, _F64P, _F64P,
                                    ctypes.c_int32, ctypes.c_int32]
        L.liberi_c_fock.argtypes = [_F64P, _F64P, ctypes.c_int32]
        L.liberi_c_finalize.argtypes = []
        L.liberi_c_last_error.argtypes = [ctypes.c_char_p, ctypes.c_int32]
        L.liberi_c_set_option.argtypes = [H, ctypes.c_char_p, ctypes.c_double]
        L.liberi_c_get_option.argtypes = [H, ctypes.c_char_p, _F64P]
        L.liberi_c_schwarz.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       _I32P, _I32P, _I32P, _I32P, _I32P,
                                       _F64P, _F64P, _F64P, _F64P, _F64P, _F64P, _F64P]
        L.liberi_c_get_stats.argtypes = [H, ctypes.POINTER(Stats)]
        L.liberi_c_quartet_fingerprint.argtypes = [H, ctypes.POINTER(ctypes.c_uint64)]
        L.liberi_c_fock_build_uhf.argtypes = [H, _F64P, _F64P, _F64P, _F64P, ctypes.c_int32]
        L.liberi_c_mdi_set_comm.argtypes = [H, H]
        L.liberi_c_comm_unique_id.argtypes = [ctypes.POINTER(ctypes.c_uint8)]
        L.liberi_c_comm_create.argtypes = [ctypes.POINTER(H), ctypes.POINTER(ctypes.c_uint8), ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32]
        L.liberi_c_comm_allreduce.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        L.liberi_c_comm_reduce_host.argtypes = [H, _F64P, _F64P, ctypes.c_int64]
        L.liberi_c_comm_destroy.argtypes = [H]
        L.liberi_c_fock_build_uhf_device.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_void_p, ctypes.c_void_p]
        L.liberi_c_setup_bytes.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                           _I32P, _I32P, _I32P, _I32P, _I32P,
                                           _F64P, _F64P, _F64P, _F64P, _F64P, _F64P, _F64P, ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_int64)]
        L.liberi_c_get_class_stats.argtypes = [H, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
        L.liberi_c_quartet_fingerprint_all.argtypes = [H, ctypes.POINTER(ctypes.c_uint64)]
        L.liberi_c_rys7_eval.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                         _F64P, _F64P]
        L.liberi_c_schwarz_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                               _I32P, _I32P, _I32P, _I32P, _I32P,
                                               _F64P, _F64P, _F64P, _F64P, _F64P, _F64P]
        L.liberi_c_rys_eval.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                        _F64P, _F64P]
        L.liberi_c_microbench.argtypes = [ctypes.c_int32, _F64P]
        L.liberi_c_rys_eval_f32.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.liberi_c_kernel_name.argtypes = [ctypes.c_int32]
        L.liberi_c_batch_create.argtypes = [ctypes.POINTER(H), ctypes.POINTER(H), ctypes.c_int32]
        L.liberi_c_batch_bind.argtypes = [H, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]
        L.liberi_c_batch_fock_build.argtypes = [H, ctypes.c_void_p]
        L.liberi_c_batch_capture.argtypes = [H]
        L.liberi_c_batch_launch.argtypes = [H, ctypes.c_void_p]
        L.liberi_c_batch_synchronize.argtypes = [H]
        L.liberi_c_batch_autotune.argtypes = [H, ctypes.c_int32, _I32P]
        L.liberi_c_batch_destroy.argtypes = [H]
        L.liberi_c_autotune.argtypes = [H, ctypes.c_int32, _I32P]
        L.liberi_c_mdi_create.argtypes = [ctypes.POINTER(H), ctypes.c_int32, ctypes.c_int32]
        L.liberi_c_mdi_payload.argtypes = [H, ctypes.c_char_p, _I32P, ctypes.POINTER(ctypes.c_int64)]
        L.liberi_c_mdi_execute.argtypes = [H, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, _I32P]
        L.liberi_c_mdi_destroy.argtypes = [H]
        L.liberi_c_set_class_variant.argtypes = [H, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        L.liberi_c_get_class_variant.argtypes = [H, ctypes.c_int32, ctypes.c_int32, _I32P]
        L.liberi_c_kernel_name.restype = ctypes.c_char_p
        for name in EXPORTS:
            if name != "liberi_c_kernel_name":
                getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        lib().liberi_c_last_error(buf, 512)
        raise LiberiError(rc, buf.value.decode(errors="replace"))


def _i32(x, keep):
    a = np.ascontiguousarray(x, dtype=np.int32)
    keep.append(a)
    return a.ctypes.data_as(_I32P)


def _f64(x, keep):
    a = np.ascontiguousarray(x, dtype=np.float64)
    keep.append(a)
    return a.ctypes.data_as(_F64P)


class LiberiHandle:
    """Opaque handle (liberi_handle_t, liberi_interface.F90:30-43)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        _check(lib().liberi_c_create(ctypes.byref(self._h)))
        self.num_bas = 0

    @property
    def ptr(self):
        return self._h

    def set_option(self, name, value):
        _check(lib().liberi_c_set_option(self._h, name.encode(), float(value)))

    def set_class_variant(self, k, precision, variant):
        """Kernel shape variant of class k (0..20) for precision 0/1."""
        _check(lib().liberi_c_set_class_variant(self._h, int(k), int(precision), int(variant)))

    def get_class_variant(self, k, precision):
        v = ctypes.c_int32()
        _check(lib().liberi_c_get_class_variant(self._h, int(k), int(precision), ctypes.byref(v)))
        return v.value

    def get_option(self, name):
        v = ctypes.c_double()
        _check(lib().liberi_c_get_option(self._h, name.encode(), ctypes.byref(v)))
        return v.value

    def stats(self):
        """Per-class arrays over all 55 classes (KERNELS_ALL: the 21 s/p/d, then
        the f block): quartets and prim_quartets of this rank; fp32_quartets and
        kernel_ms (s/p/d only, zero for the f classes)."""
        s = Stats()
        _check(lib().liberi_c_get_stats(self._h, ctypes.byref(s)))
        q, pq = np.zeros(NCLASS, dtype=np.int64), np.zeros(NCLASS, dtype=np.int64)
        pair = (ctypes.c_int64 * 2)()
        for k in range(NCLASS):
            _check(lib().liberi_c_get_class_stats(self._h, k, pair))
            q[k], pq[k] = pair[0], pair[1]
        pad = np.zeros(NCLASS - 21)
        return {"quartets": q, "fp32_quartets": np.concatenate([np.array(s.fp32_quartets[:]), pad.astype(np.int64)]),
                "prim_quartets": pq, "kernel_ms": np.concatenate([np.array(s.kernel_ms[:]), pad]),
                "build_ms": s.build_ms, "device_bytes": s.device_bytes}

    def quartet_fingerprint(self):
        """(55, 3) uint64: per class (KERNELS_ALL order) the number, sum and xor
        of the 64-bit hashes of the quartets the last build evaluated (on the
        device, over the same task lists; see liberi_c_quartet_fingerprint)."""
        out = (ctypes.c_uint64 * (3 * NCLASS))()
        _check(lib().liberi_c_quartet_fingerprint_all(self._h, out))
        return np.array(out[:], dtype=np.uint64).reshape(NCLASS, 3)

    def destroy(self):
        if self._h:
            _check(lib().liberi_c_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if self._h:
                lib().liberi_c_destroy(self._h)
        except Exception:
            pass


# ---- reference-named handle API ------------------------------------------------
def liberi_create():
    """liberi_create(handle) -- liberi_interface.F90:46-55."""
    return LiberiHandle()


def liberi_destroy(handle):
    """liberi_destroy(handle) -- cleans up if initialised (:57-70)."""
    handle.destroy()


def liberi_setup(handle, nsh, natoms, num_bas, mxgtot, ang_mom, contr_num, sh_loc, atom_num,
                 atom_loc, start_bas, end_bas, exponents, contr_coef_s, contr_coef_p, contr_coef_d,
                 contr_coef_f, coords, schwrz_int, my_rank, num_procs):
    """liberi_setup(...) -- liberi_interface.F90:72-200 (deep copy, pairs, plan)."""
    k = []
    _check(lib().liberi_c_setup(handle.ptr, nsh, natoms, num_bas, mxgtot, _i32(ang_mom, k),
                                _i32(contr_num, k), _i32(sh_loc, k), _i32(atom_num, k), _i32(atom_loc, k),
                                _i32(start_bas, k), _i32(end_bas, k), _f64(exponents, k),
                                _f64(contr_coef_s, k), _f64(contr_coef_p, k), _f64(contr_coef_d, k),
                                _f64(contr_coef_f, k), _f64(coords, k), _f64(schwrz_int, k),
                                my_rank, num_procs))
    handle.num_bas = num_bas


def liberi_fock_build(handle, density, fock, matrix_size):
    """liberi_fock_build(handle, density, fock, matrix_size) -- :202-227.
    ``fock`` (float64, C-contiguous) is overwritten with this rank's partial F."""
    d = np.ascontiguousarray(density, dtype=np.float64)
    if not (isinstance(fock, np.ndarray) and fock.dtype == np.float64 and fock.flags.c_contiguous):
        raise TypeError("fock must be a C-contiguous float64 array")
    if d.size < matrix_size or fock.size < matrix_size:
        raise LiberiError(-3, "density/fock shorter than matrix_size")
    _check(lib().liberi_c_fock_build(handle.ptr, d.ctypes.data_as(_F64P), fock.ctypes.data_as(_F64P),
                                     matrix_size))


def liberi_cleanup(handle):
    """liberi_cleanup(handle) -- :229-260."""
    _check(lib().liberi_c_cleanup(handle.ptr))


# ---- GAMESS direct-link wrapper -------------------------------------------------
def liberi_init(natoms, num_bas, nsh, mxgtot, ang_mom, contr_num, sh_loc, atom_num, atom_loc,
                start_bas, end_bas, exponents, contr_coef_s, contr_coef_p, contr_coef_d,
                contr_coef_f, coords, schwrz_int, my_rank, num_procs):
    """liberi_init (natoms first) -- gms_liberi_wrapper.F90:29-100."""
    k = []
    _check(lib().liberi_c_init(natoms, num_bas, nsh, mxgtot, _i32(ang_mom, k), _i32(contr_num, k),
                               _i32(sh_loc, k), _i32(atom_num, k), _i32(atom_loc, k), _i32(start_bas, k),
                               _i32(end_bas, k), _f64(exponents, k), _f64(contr_coef_s, k),
                               _f64(contr_coef_p, k), _f64(contr_coef_d, k), _f64(contr_coef_f, k),
                               _f64(coords, k), _f64(schwrz_int, k), my_rank, num_procs))


def liberi_fock(density, fock, n):
    """liberi_fock(density, fock, n) with the wrapper's size check -- :103-131."""
    d = np.ascontiguousarray(density, dtype=np.float64)
    _check(lib().liberi_c_fock(d.ctypes.data_as(_F64P), fock.ctypes.data_as(_F64P), n))


def liberi_finalize():
    """liberi_finalize() -- :134-146."""
    _check(lib().liberi_c_finalize())


# ---- conveniences over a basis dict ---------------------------------------------
def _basis_args(b):
    nsh = int(b["nsh"])
    mx = int(b["mxgtot"])
    z = np.zeros(nsh * mx)
    return (nsh, int(b["natoms"]), int(b["num_bas"]), mx, b["ang_mom"], b["contr_num"], b["sh_loc"],
            b["atom_num"], b["atom_loc"], b.get("start_bas", b["atom_loc"]), b.get("end_bas", b["atom_loc"]),
            b["exponents"], b["coef_s"], b["coef_p"], b["coef_d"], b.get("coef_f", z), b["coords"])


def setup_from_basis(handle, basis, schwrz=None, my_rank=0, num_procs=1):
    (nsh, natoms, nbf, mx, ang, cn, sl, an, al, sb, eb, ex, cs, cp, cd, cf, xyz) = _basis_args(basis)
    sw = basis["schwrz"] if schwrz is None else schwrz
    liberi_setup(handle, nsh, natoms, nbf, mx, ang, cn, sl, an, al, sb, eb, ex, cs, cp, cd, cf, xyz, sw,
                 my_rank, num_procs)


def fock(handle, density):
    """Packed partial F for packed D through liberi_fock_build."""
    n = handle.num_bas
    ntri = n * (n + 1) // 2
    out = np.zeros(ntri)
    liberi_fock_build(handle, density, out, ntri)
    return out


def fock_uhf(handle, density_a, density_b):
    """Open-shell partials (F_alpha, F_beta) = (J(Da+Db) - K(2 Da), J(Da+Db) - K(2 Db)) for packed
    alpha and beta densities (liberi_c_fock_build_uhf); Da = Db = D/2 gives the closed-shell F."""
    n = handle.num_bas
    ntri = n * (n + 1) // 2
    da = np.ascontiguousarray(density_a, dtype=np.float64)
    db = np.ascontiguousarray(density_b, dtype=np.float64)
    if da.shape != (ntri,) or db.shape != (ntri,):
        raise ValueError("densities must be packed of length %d" % ntri)
    fa, fb = np.zeros(ntri), np.zeros(ntri)
    _check(lib().liberi_c_fock_build_uhf(handle._h, da.ctypes.data_as(_F64P), db.ctypes.data_as(_F64P),
                                         fa.ctypes.data_as(_F64P), fb.ctypes.data_as(_F64P), ntri))
    return fa, fb


def microbench(kind):
    """0: FP64 FMA TFLOP/s, 1: FP32 FMA TFLOP/s, 2: FP64 atomicAdd Gatomic/s."""
    v = ctypes.c_double()
    _check(lib().liberi_c_microbench(kind, ctypes.byref(v)))
    return v.value


def fock_build_device(handle, d_density_ptr, d_fock_ptr, stream_ptr=0):
    """liberi_c_fock_build_device on raw device pointers (enqueued, async)."""
    _check(lib().liberi_c_fock_build_device(handle.ptr, ctypes.c_void_p(d_density_ptr),
                                            ctypes.c_void_p(d_fock_ptr), ctypes.c_void_p(stream_ptr)))


def autotune(handle, reps=3):
    """Per-class kets-per-task choice timed on the handle's device buffers."""
    out = np.zeros(21, dtype=np.int32)
    _check(lib().liberi_c_autotune(handle.ptr, int(reps), out.ctypes.data_as(_I32P)))
    return out


class Batch:
    """Several set-up handles built together: one launch per class over all
    molecules, optionally captured once as a CUDA graph (liberi_c_batch_*)."""

    def __init__(self, handles):
        self.handles = list(handles)
        arr = (ctypes.c_void_p * len(self.handles))(*[h.ptr.value for h in self.handles])
        self._b = ctypes.c_void_p()
        _check(lib().liberi_c_batch_create(ctypes.byref(self._b), arr, len(self.handles)))

    def bind(self, d_density_ptrs, d_fock_ptrs):
        n = len(self.handles)
        dp = (ctypes.c_void_p * n)(*d_density_ptrs)
        fp = (ctypes.c_void_p * n)(*d_fock_ptrs)
        _check(lib().liberi_c_batch_bind(self._b, dp, fp))

    def fock_build(self, stream_ptr=0):
        _check(lib().liberi_c_batch_fock_build(self._b, ctypes.c_void_p(stream_ptr)))

    def capture(self):
        _check(lib().liberi_c_batch_capture(self._b))

    def launch(self, stream_ptr=0):
        _check(lib().liberi_c_batch_launch(self._b, ctypes.c_void_p(stream_ptr)))

    def synchronize(self):
        _check(lib().liberi_c_batch_synchronize(self._b))

    def autotune(self, reps=3):
        out = np.zeros(21, dtype=np.int32)
        _check(lib().liberi_c_batch_autotune(self._b, int(reps), out.ctypes.data_as(_I32P)))
        return out

    def destroy(self):
        if self._b:
            _check(lib().liberi_c_batch_destroy(self._b))
            self._b = ctypes.c_void_p()


class MDIEngine:
    """The MDI plugin's command set (liberi_c_mdi_*): `send(cmd, data)` for
    '>' commands, `recv(cmd)` for '<' commands, `command(cmd)` for the rest;
    returns or raises like the C ABI.  A driver emulation for tests and for
    Python front ends of the plugin."""

    TYPES = {1: np.int32, 2: np.float64, 3: np.uint8}

    def __init__(self, rank=0, nprocs=1):
        self._s = ctypes.c_void_p()
        _check(lib().liberi_c_mdi_create(ctypes.byref(self._s), int(rank), int(nprocs)))
        self.terminated = False

    def payload(self, cmd):
        t = ctypes.c_int32()
        n = ctypes.c_int64()
        _check(lib().liberi_c_mdi_payload(self._s, cmd.encode(), ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    def _run(self, cmd, buf, count):
        term = ctypes.c_int32()
        ptr = None if buf is None else buf.ctypes.data_as(ctypes.c_void_p)
        _check(lib().liberi_c_mdi_execute(self._s, cmd.encode(), ptr, int(count), ctypes.byref(term)))
        self.terminated = bool(term.value)

    def send(self, cmd, data):
        t, n = self.payload(cmd)
        if t == 3:
            buf = np.frombuffer(data.ljust(n)[:n].encode(), dtype=np.uint8).copy()
        else:
            buf = np.ascontiguousarray(np.atleast_1d(data), dtype=self.TYPES[t])
        self._run(cmd, buf, buf.size)

    def recv(self, cmd):
        t, n = self.payload(cmd)
        buf = np.zeros(n, dtype=self.TYPES[t])
        self._run(cmd, buf, n)
        return buf

    def command(self, cmd):
        self._run(cmd, None, 0)

    def set_comm(self, comm):
        """Sum the ranks' partial F over `comm` (a Comm, or None) inside '<FOCK'."""
        _check(lib().liberi_c_mdi_set_comm(self._s, comm._c if comm is not None else None))

    def destroy(self):
        if self._s:
            _check(lib().liberi_c_mdi_destroy(self._s))
            self._s = ctypes.c_void_p()


class Comm:
    """NCCL communicator for the sum of the ranks' partial F (liberi_c_comm_*).
    Rank 0 calls `unique_id()`, the caller broadcasts the bytes, every rank
    constructs `Comm(uid, rank, nranks, device)` (waits for all ranks)."""

    ID_BYTES = 128

    @staticmethod
    def unique_id():
        buf = (ctypes.c_uint8 * Comm.ID_BYTES)()
        _check(lib().liberi_c_comm_unique_id(buf))
        return bytes(buf)

    def __init__(self, uid, rank=0, nranks=1, device=-1):
        self._c = ctypes.c_void_p()
        buf = (ctypes.c_uint8 * Comm.ID_BYTES).from_buffer_copy(uid)
        _check(lib().liberi_c_comm_create(ctypes.byref(self._c), buf, int(rank), int(nranks), int(device)))

    def allreduce_device(self, d_send, d_recv, count, stream=None):
        _check(lib().liberi_c_comm_allreduce(self._c, d_send, d_recv, int(count), stream))

    def reduce_host(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.empty_like(x)
        _check(lib().liberi_c_comm_reduce_host(self._c, x.ctypes.data_as(_F64P), out.ctypes.data_as(_F64P), x.size))
        return out

    def destroy(self):
        if self._c:
            _check(lib().liberi_c_comm_destroy(self._c))
            self._c = ctypes.c_void_p()


def rys_eval(n, T, thr=60.0, strict=False):
    """Engine Rys roots/weights (host evaluation of the device tables)."""
    u = np.zeros(n)
    w = np.zeros(n)
    _check(lib().liberi_c_rys_eval(n, T, thr, int(strict), u.ctypes.data_as(_F64P), w.ctypes.data_as(_F64P)))
    return u, w


def rys7_eval(n, T, thr=65.0, strict=False):
    """The f classes' Rys roots/weights, n = 1..7 (host evaluation of their table)."""
    u = np.zeros(n)
    w = np.zeros(n)
    _check(lib().liberi_c_rys7_eval(n, T, thr, int(strict), u.ctypes.data_as(_F64P), w.ctypes.data_as(_F64P)))
    return u, w


def rys_eval_f32(n, T, thr=60.0, strict=False):
    """FP32-tier Rys roots/weights (host evaluation in single precision)."""
    u = np.zeros(n, dtype=np.float32)
    w = np.zeros(n, dtype=np.float32)
    FP = ctypes.POINTER(ctypes.c_float)
    _check(lib().liberi_c_rys_eval_f32(n, T, thr, int(strict), u.ctypes.data_as(FP), w.ctypes.data_as(FP)))
    return u.astype(np.float64), w.astype(np.float64)


def setup_bytes(basis, schwarz_cut=5.00000000000000018e-11):
    """Device bytes liberi_setup would allocate for `basis` (host-only dry run)."""
    (nsh, natoms, nbf, mx, ang, cn, sl, an, al, sb, eb, ex, cs, cp, cd, cf, xyz) = _basis_args(basis)
    k = []
    out = ctypes.c_int64()
    _check(lib().liberi_c_setup_bytes(nsh, natoms, nbf, mx, _i32(ang, k), _i32(cn, k), _i32(sl, k), _i32(an, k),
                                      _i32(al, k), _f64(ex, k), _f64(cs, k), _f64(cp, k), _f64(cd, k),
                                      _f64(cf, k), _f64(xyz, k), _f64(basis["schwrz"], k), float(schwarz_cut),
                                      ctypes.byref(out)))
    return int(out.value)


def schwarz(basis):
    """Packed shell Schwarz table computed on the device."""
    (nsh, natoms, nbf, mx, ang, cn, sl, an, al, sb, eb, ex, cs, cp, cd, cf, xyz) = _basis_args(basis)
    k = []
    out = np.zeros(nsh * (nsh + 1) // 2)
    _check(lib().liberi_c_schwarz(nsh, natoms, nbf, mx, _i32(ang, k), _i32(cn, k), _i32(sl, k),
                                  _i32(an, k), _i32(al, k), _f64(ex, k), _f64(cs, k), _f64(cp, k),
                                  _f64(cd, k), _f64(cf, k), _f64(xyz, k), out.ctypes.data_as(_F64P)))
    return out


def schwarz_noalloc(basis):
    """Packed shell Schwarz table without any device allocation.

    For callers that cannot call cudaMalloc: their device memory is already
    committed to their own pool, or their allocation policy forbids ad-hoc
    cudaMalloc/cudaFree.  The engine's device working memory for this call is
    a fixed 8 MiB array, committed by the first call on each device (make that
    call at start-up, before a pool claims the memory); bases that need more
    raise LiberiError (LIBERI_E_NOMEM) and should use schwarz() instead."""
    (nsh, natoms, nbf, mx, ang, cn, sl, an, al, sb, eb, ex, cs, cp, cd, cf, xyz) = _basis_args(basis)
    k = []
    out = np.zeros(nsh * (nsh + 1) // 2)
    _check(lib().liberi_c_schwarz_noalloc(nsh, natoms, nbf, mx, _i32(ang, k), _i32(cn, k), _i32(sl, k),
                                          _i32(an, k), _i32(al, k), _f64(ex, k), _f64(cs, k), _f64(cp, k),
                                          _f64(cd, k), _f64(xyz, k), out.ctypes.data_as(_F64P)))
    return out
