"""ctypes front end of the CPU oracle (oracle/liberi_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py's CPU-baseline leg.  The product never imports it.

A basis is a dict with the reference's liberi_setup arrays
(src/interface/liberi_interface.F90:72-200): nsh, natoms, num_bas, mxgtot,
ang_mom, contr_num, sh_loc, atom_num, atom_loc, start_bas, end_bas, exponents,
coef_s, coef_p, coef_d, coef_f, coords, schwrz.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libliberi_oracle.so")

KERNELS = ["int0000", "int0001", "int0011", "int0111", "int0101", "int1111",
           "int0002", "int0012", "int0102", "int0112", "int0022", "int0122",
           "int1102", "int0202", "int2211", "int2121", "int2120", "int2111",
           "int2220", "int2221", "int2222"]
# the f block of the driver, in its order (src/liberi_driver.F90:103-160)
KERNELS_F = ["int3333", "int0030", "int0031", "int0032", "int1030", "int3330", "int3011", "int3020",
             "int2130", "int2230", "int3030", "int3110", "int3111", "int3120", "int3121", "int2231",
             "int3130", "int3131", "int3210", "int3331", "int3211", "int3220", "int3221", "int3222",
             "int3230", "int3231", "int3232", "int3300", "int3310", "int3311", "int3320", "int3321",
             "int3322", "int3332"]
NK = len(KERNELS) + len(KERNELS_F)

_I32P = ctypes.POINTER(ctypes.c_int32)
_F64P = ctypes.POINTER(ctypes.c_double)


class _Basis(ctypes.Structure):
    _fields_ = [("nsh", ctypes.c_int32), ("natoms", ctypes.c_int32),
                ("num_bas", ctypes.c_int32), ("mxgtot", ctypes.c_int32),
                ("ang_mom", _I32P), ("contr_num", _I32P), ("sh_loc", _I32P),
                ("atom_num", _I32P), ("atom_loc", _I32P),
                ("exponents", _F64P), ("coef_s", _F64P), ("coef_p", _F64P),
                ("coef_d", _F64P), ("coef_f", _F64P), ("coords", _F64P), ("schwrz", _F64P)]


class _Opts(ctypes.Structure):
    _fields_ = [("schwarz_cut", ctypes.c_double), ("eri_cut", ctypes.c_double),
                ("my_rank", ctypes.c_int32), ("num_procs", ctypes.c_int32),
                ("sample_mod", ctypes.c_int32), ("sample_seed", ctypes.c_int32),
                ("nthreads", ctypes.c_int32), ("only_kernel", ctypes.c_int32)]


class _Counts(ctypes.Structure):
    _fields_ = [("c", (ctypes.c_int64 * 4) * NK), ("t_wall", ctypes.c_double * NK),
                ("t_eval", ctypes.c_double * NK), ("nthreads", ctypes.c_int32),
                ("fp", (ctypes.c_uint64 * 2) * NK), ("ops", (ctypes.c_uint64 * 2) * NK)]


_lib = None
_oplib = None
_OPCOUNT_PATH = os.path.join(_HERE, "_build", "liberi_opcount.so")


def build():
    """Compile the oracle with its Makefile (gcc -O2 -fopenmp)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.oracle_fock_build.argtypes = [ctypes.POINTER(_Basis), ctypes.POINTER(_Opts),
                                           _F64P, _F64P, ctypes.POINTER(_Counts)]
        _lib.oracle_fock_build.restype = ctypes.c_int
        _lib.oracle_fock_build_jk.argtypes = [ctypes.POINTER(_Basis), ctypes.POINTER(_Opts),
                                              _F64P, _F64P, _F64P, ctypes.POINTER(_Counts)]
        _lib.oracle_fock_build_jk.restype = ctypes.c_int
        _lib.oracle_schwarz.argtypes = [ctypes.POINTER(_Basis), _F64P]
        _lib.oracle_schwarz.restype = ctypes.c_int
        _lib.oracle_rys_roots.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, _F64P, _F64P]
        _lib.oracle_rys_roots.restype = None
        _lib.oracle_rys_roots_grid.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_int, ctypes.c_int, _F64P, _F64P]
        _lib.oracle_rys_roots_grid.restype = None
        _lib.oracle_rank_owns.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                          ctypes.c_int, ctypes.c_int]
        _lib.oracle_rank_owns.restype = ctypes.c_int
    return _lib


def _basis_struct(b, keep):
    def i32(name):
        a = np.ascontiguousarray(b[name], dtype=np.int32)
        keep.append(a)
        return a.ctypes.data_as(_I32P)

    def f64(name):
        v = b[name] if name in b else np.zeros(len(b["exponents"]))  # bases without f: no coef_f
        a = np.ascontiguousarray(v, dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(_F64P)

    return _Basis(int(b["nsh"]), int(b["natoms"]), int(b["num_bas"]), int(b["mxgtot"]),
                  i32("ang_mom"), i32("contr_num"), i32("sh_loc"), i32("atom_num"),
                  i32("atom_loc"), f64("exponents"), f64("coef_s"), f64("coef_p"),
                  f64("coef_d"), f64("coef_f"), f64("coords"), f64("schwrz"))


def fock_build(basis, density, *, schwarz_cut=5e-11, eri_cut=5e-11, my_rank=0,
               num_procs=1, sample_mod=1, sample_seed=0, nthreads=0, only_kernel=-1,
               return_counts=False, return_times=False, return_info=False):
    """Packed F (this rank's partial) for packed D; optional per-kernel counts
    [screened quartets, primitive quartets, digested integrals, evaluated] and
    times (wall seconds per kernel, evaluation seconds summed over threads,
    thread count), one row per kernel: the 21 s/p/d kernels, then the 34 of
    the f block (KERNELS + KERNELS_F).  return_info: (F, dict) with "counts",
    "t_wall", "t_eval", "nthreads" and "fingerprint", an (NK, 3) uint64 array
    per kernel of the screened-quartet set [count, sum, xor] (see quartet_fp in
    the C file)."""
    keep = []
    bs = _basis_struct(basis, keep)
    n = int(basis["num_bas"])
    d = np.ascontiguousarray(density, dtype=np.float64)
    assert d.shape == (n * (n + 1) // 2,)
    f = np.zeros_like(d)
    opts = _Opts(schwarz_cut, eri_cut, my_rank, num_procs, sample_mod, sample_seed,
                 nthreads, only_kernel)
    cnt = _Counts()
    rc = lib().oracle_fock_build(ctypes.byref(bs), ctypes.byref(opts),
                                 d.ctypes.data_as(_F64P), f.ctypes.data_as(_F64P),
                                 ctypes.byref(cnt))
    if rc != 0:
        raise RuntimeError("oracle_fock_build failed: %d" % rc)
    counts = np.array([[cnt.c[k][j] for j in range(4)] for k in range(NK)], dtype=np.int64)
    if return_info:
        fp = np.zeros((NK, 3), dtype=np.uint64)
        for k in range(NK):
            fp[k] = (np.uint64(counts[k, 0]), np.uint64(cnt.fp[k][0]), np.uint64(cnt.fp[k][1]))
        return f, {"counts": counts, "t_wall": np.array(cnt.t_wall[:]), "t_eval": np.array(cnt.t_eval[:]),
                   "nthreads": int(cnt.nthreads), "fingerprint": fp}
    if return_times:
        return f, counts, (np.array(cnt.t_wall[:]), np.array(cnt.t_eval[:]), int(cnt.nthreads))
    if return_counts:
        return f, counts
    return f


def count_ops(basis, density, *, schwarz_cut=5e-11, eri_cut=5e-11, sample_mod=1, sample_seed=0,
              nthreads=0):
    """Floating-point operations of this restatement of the reference
    algorithm, per class, from the op-counting build (oracle/opcount.cpp) on
    a hashed 1/sample_mod sample of the screened quartets: an (NK, 4) array of
    [operations in primitive-quartet work, operations in shell-quartet work,
    primitive quartets evaluated, shell quartets evaluated]."""
    global _oplib
    if _oplib is None:
        if not os.path.exists(_OPCOUNT_PATH):
            build()
        _oplib = ctypes.CDLL(_OPCOUNT_PATH)
        _oplib.oracle_fock_build.argtypes = lib().oracle_fock_build.argtypes
        _oplib.oracle_fock_build.restype = ctypes.c_int
    keep = []
    bs = _basis_struct(basis, keep)
    n = int(basis["num_bas"])
    d = np.ascontiguousarray(density, dtype=np.float64)
    assert d.shape == (n * (n + 1) // 2,)
    f = np.zeros_like(d)
    opts = _Opts(schwarz_cut, eri_cut, 0, 1, sample_mod, sample_seed, nthreads, -1)
    cnt = _Counts()
    rc = _oplib.oracle_fock_build(ctypes.byref(bs), ctypes.byref(opts), d.ctypes.data_as(_F64P),
                                  f.ctypes.data_as(_F64P), ctypes.byref(cnt))
    if rc != 0:
        raise RuntimeError("oracle op count failed: %d" % rc)
    return np.array([[cnt.ops[k][0], cnt.ops[k][1], cnt.c[k][1], cnt.c[k][3]] for k in range(NK)],
                    dtype=np.float64)


def fock_build_uhf(basis, density_a, density_b, **kw):
    """Open-shell partials (F_alpha, F_beta) = (J(Da + Db) - K(2 Da), J(Da + Db) - K(2 Db)) in the
    units of fock_build; keyword options as fock_build (no counts)."""
    out = []
    for ds in (density_a, density_b):
        out.append(_build_jk(basis, np.asarray(density_a) + np.asarray(density_b), 2.0 * np.asarray(ds), **kw))
    return out[0], out[1]


def _build_jk(basis, dj, dk, *, schwarz_cut=5e-11, eri_cut=5e-11, my_rank=0, num_procs=1, nthreads=0):
    keep = []
    bs = _basis_struct(basis, keep)
    n = int(basis["num_bas"])
    dj = np.ascontiguousarray(dj, dtype=np.float64)
    dk = np.ascontiguousarray(dk, dtype=np.float64)
    assert dj.shape == dk.shape == (n * (n + 1) // 2,)
    f = np.zeros_like(dj)
    opts = _Opts(schwarz_cut, eri_cut, my_rank, num_procs, 1, 0, nthreads, -1)
    cnt = _Counts()
    rc = lib().oracle_fock_build_jk(ctypes.byref(bs), ctypes.byref(opts), dj.ctypes.data_as(_F64P),
                                    dk.ctypes.data_as(_F64P), f.ctypes.data_as(_F64P), ctypes.byref(cnt))
    if rc != 0:
        raise RuntimeError("oracle_fock_build_jk failed: %d" % rc)
    return f


def schwarz(basis):
    """Packed Schwarz table sqrt(max |(ab|ab)|) over shells."""
    keep = []
    b = dict(basis)
    nsh = int(b["nsh"])
    b["schwrz"] = np.ones(nsh * (nsh + 1) // 2)
    bs = _basis_struct(b, keep)
    out = np.zeros(nsh * (nsh + 1) // 2)
    lib().oracle_schwarz(ctypes.byref(bs), out.ctypes.data_as(_F64P))
    return out


def rys_roots(n, T, thr=55.0, rot=False, ngrid=None):
    """Roots and weights of the oracle's rule: the reference's grid for n roots
    (30 points up to 4, 35 for 5, 40 for 6 and 7) unless ngrid is given."""
    u = np.zeros(n)
    w = np.zeros(n)
    if ngrid is None:
        lib().oracle_rys_roots(n, T, thr, int(rot), u.ctypes.data_as(_F64P), w.ctypes.data_as(_F64P))
    else:
        lib().oracle_rys_roots_grid(n, T, thr, int(rot), int(ngrid), u.ctypes.data_as(_F64P),
                                    w.ctypes.data_as(_F64P))
    return u, w


def rank_owns(tile, ntot, it, rank, nsize):
    return bool(lib().oracle_rank_owns(tile, ntot, it, rank, nsize))
