"""The allocation-free Schwarz entry point (liberi_c_schwarz_noalloc).

Some callers cannot call cudaMalloc: their device memory is already committed
to their own pool allocator, or their allocation policy forbids ad-hoc
cudaMalloc/cudaFree because those calls synchronise the device.  For them the
library offers a Schwarz-table generator whose device working memory is a
fixed array, committed by the first call on each device.  This file checks,
through the C ABI, that two calls in a row return what the allocating entry
point (liberi_c_schwarz) and the CPU oracle return, that a call after the
first leaves the device's free memory unchanged, and that a basis too large
for the fixed array is refused with a clear error.  It is named so that
pytest collects it last.
"""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from oracle import oracle

pytestmark = pytest.mark.gpu

# same kernels on the same inputs as the allocating entry point: the tables
# agree to rounding; against the oracle (Rys roots from the reference's
# Stieltjes procedure instead of the engine's tables) to the parity bar
RTOL_SAME = 1e-12
RTOL_ORACLE = 1e-10


def test_noalloc_schwarz_matches_allocating_entry_point_and_oracle_twice():
    # two calls in a row: the array keeps the previous call's contents
    for basis in (M.ethane(), M.random_molecule(7, seed=2)):
        ref = liberi.schwarz(basis)
        ora = oracle.schwarz(basis)
        got = liberi.schwarz_noalloc(basis)
        assert got.shape == ref.shape == ora.shape
        assert np.allclose(got, ref, rtol=RTOL_SAME, atol=1e-300), np.abs(got - ref).max()
        assert np.allclose(got, ora, rtol=RTOL_ORACLE, atol=1e-14), np.abs(got - ora).max()
        assert np.all(got >= 0.0)


def test_noalloc_schwarz_allocates_no_device_memory():
    import torch

    basis = M.random_molecule(9, seed=4)
    first = liberi.schwarz_noalloc(basis)  # commits the array on this device
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    second = liberi.schwarz_noalloc(basis)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.array_equal(first, second)


def test_noalloc_schwarz_rejects_bases_over_the_limit():
    # 60 carbon atoms at one point keep all 405,000 primitive pairs (~19 MB of
    # device data, above the 8 MiB array); the check happens before any GPU work
    basis = M.c60()
    basis["coords"] = np.zeros_like(basis["coords"])
    with pytest.raises(liberi.LiberiError) as e:
        liberi.schwarz_noalloc(basis)
    assert e.value.code == -5
    assert "limit" in str(e.value)
