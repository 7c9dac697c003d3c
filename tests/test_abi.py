"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/liberi_b200.h, and rejects misuse before touching the
device (the reference's `error stop 1` paths, liberi_interface.F90:219-222,
gms_liberi_wrapper.F90:117-127)."""
import os
import re

import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from conftest import ROOT


def test_header_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "liberi_b200.h")).read()
    declared = set(re.findall(r"\b(liberi_c_\w+)\s*\(", hdr))
    assert len(declared) >= 15
    L = liberi.lib()
    for name in declared:
        assert hasattr(L, name), name
    assert set(liberi.EXPORTS) == declared


def test_kernel_names_in_driver_order():
    L = liberi.lib()
    names = [L.liberi_c_kernel_name(i).decode() for i in range(55)]
    assert names == liberi.KERNELS_ALL  # the s/p/d kernels, then the f block
    assert L.liberi_c_kernel_name(55) is None
    from oracle import oracle
    assert liberi.KERNELS_ALL == oracle.KERNELS + oracle.KERNELS_F


def test_fock_before_setup_is_state_error():
    h = liberi.liberi_create()
    with pytest.raises(liberi.LiberiError) as e:
        liberi.liberi_fock_build(h, np.zeros(1), np.zeros(1), 1)
    assert e.value.code == -2
    liberi.liberi_cleanup(h)   # cleanup of an uninitialised handle is a no-op
    liberi.liberi_cleanup(h)
    liberi.liberi_destroy(h)


def test_wrapper_before_init_is_state_error():
    liberi.liberi_finalize()
    with pytest.raises(liberi.LiberiError) as e:
        liberi.liberi_fock(np.zeros(3), np.zeros(3), 3)
    assert e.value.code == -2


def test_options_validate():
    h = liberi.liberi_create()
    assert h.get_option("schwarz_cut") == pytest.approx(5e-11)
    assert h.get_option("eri_cut") == pytest.approx(5e-11)
    h.set_option("precision", 1)
    assert h.get_option("precision") == 1
    # FP32-tier primitive screening: default 1e-8 of the cut, 0 disables
    assert h.get_option("fp32_prim") == pytest.approx(1e-8)
    h.set_option("fp32_prim", 0.0)
    assert h.get_option("fp32_prim") == 0.0
    for name, val in [("nope", 1.0), ("precision", 2), ("schwarz_cut", -1.0), ("fp32_prim", -1.0),
                      ("fp32_prim", 2.0)]:
        with pytest.raises(liberi.LiberiError) as e:
            h.set_option(name, val)
        assert e.value.code == -1


def test_launch_options_round_trip():
    # the scheduling and tiling options: defaults, set/get, rejected values
    h = liberi.liberi_create()
    assert h.get_option("overlap") == 1 and h.get_option("fan") == 1
    assert h.get_option("tile_mask") == 0 and h.get_option("rank_split") == 0
    # FP64 side stream: (ss|dd), (sp|dd), (sd|sd) and the seven Rys classes
    side = [liberi.KERNELS.index(n) for n in ("int0022", "int0122", "int0202", "int2211", "int2121", "int2120",
                                               "int2111", "int2220", "int2221", "int2222")]
    assert h.get_option("side_mask") == sum(1 << k for k in side)
    for name, val in [("overlap", 0), ("fan", 0), ("tile_mask", 5), ("rank_split", 1), ("side_mask", 0)]:
        h.set_option(name, val)
        assert h.get_option(name) == val
    for name, val in [("tile_mask", -1), ("tile_mask", float(1 << 21)), ("rank_split", 2), ("side_mask", -1),
                      ("side_mask", float(1 << 21))]:
        with pytest.raises(liberi.LiberiError) as e:
            h.set_option(name, val)
        assert e.value.code == -1
    liberi.liberi_destroy(h)


@pytest.mark.parametrize("bad", ["gshell", "fshell_size", "rank", "sizes", "num_bas"])
def test_setup_rejects_bad_input(bad):
    h = liberi.liberi_create()
    args = dict(nsh=1, natoms=1, num_bas=1, mxgtot=1, ang=[1], rank=0, nproc=1)
    if bad == "gshell":  # ang_mom 5 (g) is beyond the reference's kernels
        args["ang"] = [5]
        code = -1
    elif bad == "fshell_size":  # an f shell's ten functions do not fit num_bas = 1
        args["ang"] = [4]
        code = -1
    elif bad == "num_bas":
        # n(n+1)/2 of 65536 functions exceeds the int32 matrix_size
        args["num_bas"] = 65536
        code = -6
    elif bad == "rank":
        args["rank"] = 3
        args["nproc"] = 2
        code = -1
    else:
        args["nsh"] = 0
        code = -1
    with pytest.raises(liberi.LiberiError) as e:
        liberi.liberi_setup(h, args["nsh"], args["natoms"], args["num_bas"], args["mxgtot"], args["ang"],
                            [1], [1], [1], [1], [1], [1], [1.0], [1.0], [0.0], [0.0], [0.0],
                            [0.0, 0.0, 0.0], [1.0], args["rank"], args["nproc"])
    assert e.value.code == code


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_engine_rys_tables_match_oracle(n):
    # the piecewise tables reproduce the Stieltjes roots: the oracle's 40-point
    # rule on the whole table range, the reference's own grid for n roots
    # (30 points up to 4, 35 for 5) below that class's threshold
    from oracle import oracle
    rng = np.random.default_rng(n)
    thr_ref = {1: 43.0, 2: 43.0, 3: 43.0, 4: 49.0, 5: 55.0}[n]
    for T in np.concatenate([[0.0, 1e-9, 0.5, 24.999, 25.0, 42.99, 59.9], rng.uniform(0, 60, 40)]):
        ue, we = liberi.rys_eval(n, float(T), thr=60.0)
        uo, wo = oracle.rys_roots(n, float(T), thr=60.0, ngrid=40)
        assert np.allclose(ue, uo, rtol=5e-13, atol=0), (n, T)
        assert np.allclose(we, wo, rtol=5e-13, atol=0), (n, T)
        if T < thr_ref:
            ur, wr = oracle.rys_roots(n, float(T), thr=thr_ref)
            assert np.allclose(ue, ur, rtol=5e-13, atol=0), (n, T)
            assert np.allclose(we, wr, rtol=5e-13, atol=0), (n, T)
    for T in [25.5, 70.0, 300.0]:
        ue, we = liberi.rys_eval(n, T, thr=25.0, strict=True)
        uo, wo = oracle.rys_roots(n, T, thr=25.0, rot=True)
        assert np.allclose(ue, uo, rtol=1e-14) and np.allclose(we, wo, rtol=1e-14)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7])
def test_engine_rys7_tables_match_oracle(n):
    # the f classes' table (1..7 roots on [0, 65)) against the oracle's 40-point rule
    from oracle import oracle
    rng = np.random.default_rng(100 + n)
    for T in np.concatenate([[0.0, 1e-9, 0.5, 24.999, 25.0, 42.99, 59.9, 64.9], rng.uniform(0, 65, 40)]):
        ue, we = liberi.rys7_eval(n, float(T), thr=65.0)
        uo, wo = oracle.rys_roots(n, float(T), thr=65.0, ngrid=40)
        assert np.allclose(ue, uo, rtol=5e-13, atol=0), (n, T, ue, uo)
        assert np.allclose(we, wo, rtol=5e-13, atol=0), (n, T, we, wo)
    for T in [25.5, 70.0, 300.0]:
        ue, we = liberi.rys7_eval(n, T, thr=25.0, strict=True)
        uo, wo = oracle.rys_roots(n, T, thr=25.0, rot=True)
        assert np.allclose(ue, uo, rtol=1e-14) and np.allclose(we, wo, rtol=1e-14)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_engine_fp32_rys_tables(n):
    # the FP32 tier's tables, evaluated in single precision as on the device:
    # relative error within a few float ulps of the reference roots/weights
    from oracle import oracle
    rng = np.random.default_rng(100 + n)
    worst = 0.0
    for T in np.concatenate([[0.0, 1e-6, 0.25, 0.5, 24.999, 42.99, 59.99], rng.uniform(0, 60, 200)]):
        uf, wf = liberi.rys_eval_f32(n, float(T), thr=60.0)
        uo, wo = oracle.rys_roots(n, float(np.float32(T)), thr=60.0)
        worst = max(worst, np.max(np.abs(uf - uo) / np.abs(uo)), np.max(np.abs(wf - wo) / np.abs(wo)))
    assert worst <= 3e-6, worst


def test_class_variant_arguments():
    # shape variants are per class (0..20), per precision (0 FP64, 1 FP32), 0..2
    h = liberi.liberi_create()
    assert h.get_class_variant(5, 0) == 0 and h.get_class_variant(5, 1) == 0
    h.set_class_variant(5, 1, 2)
    assert h.get_class_variant(5, 1) == 2 and h.get_class_variant(5, 0) == 0
    for bad in ((21, 0, 0), (-1, 0, 0), (0, 2, 0), (0, 0, 3), (0, 0, -1)):
        with pytest.raises(liberi.LiberiError) as e:
            h.set_class_variant(*bad)
        assert e.value.code == -1
    liberi.liberi_destroy(h)


def test_fortran_shim_matches_the_c_abi():
    """The Fortran iso_c_binding shim (shipped as source: no Fortran compiler
    here) binds only functions the header declares and the library exports,
    each with the header's number of arguments."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, "gms_liberi_b200", "fortran", "liberi_b200_interface.F90")).read()
    src = re.sub(r"&\s*\n\s*", " ", src)  # join continuation lines
    header = open(os.path.join(root, "include", "liberi_b200.h")).read()
    binds = re.findall(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", src, re.I)
    assert len(binds) >= 6
    lib = liberi.lib()
    for fname, args, cname in binds:
        assert fname == cname
        m = re.search(r"\bint\s+%s\s*\(([^)]*)\)\s*;" % cname, header, re.S)
        assert m, cname
        n_c = 0 if m.group(1).strip() in ("", "void") else len(m.group(1).split(","))
        n_f = 0 if not args.strip() else len(args.split(","))
        assert n_f == n_c, (cname, n_f, n_c)
        assert hasattr(lib, cname), cname


def test_device_memory_limit_fails_setup_before_device_work():
    # an allocation failure made on the host: the handle's byte limit is
    # checked by the host half of setup, before any CUDA call, so this runs
    # without a GPU and leaves the handle usable
    b = M.ethane()
    b["schwrz"] = np.ones(b["nsh"] * (b["nsh"] + 1) // 2)
    h = liberi.liberi_create()
    h.set_option("max_device_bytes", 1000.0)
    assert h.get_option("max_device_bytes") == 1000.0
    with pytest.raises(liberi.LiberiError) as e:
        liberi.setup_from_basis(h, b)
    assert e.value.code == -5 and "max_device_bytes" in str(e.value)
    need = liberi.setup_bytes(b, 5e-11)
    assert need > 1000
    with pytest.raises(liberi.LiberiError) as e:
        h.set_option("max_device_bytes", -1.0)
    assert e.value.code == -1
    liberi.liberi_destroy(h)


def test_double_cleanup_and_destroy():
    # liberi_cleanup on a handle that is not set up is a no-op
    # (liberi_interface.F90:236), also twice in a row; destroy after cleanup
    h = liberi.liberi_create()
    liberi.liberi_cleanup(h)
    liberi.liberi_cleanup(h)
    liberi.liberi_destroy(h)
