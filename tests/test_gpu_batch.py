"""Batched builds of several molecules (liberi_c_batch_*) and the per-class
autotuner: each molecule's F from one batched launch sequence, from a
captured CUDA graph and after autotuning must equal its own single-molecule
build (same quartets, same digestion; only the order of FP64 atomics
differs) and the oracle within the FP64 parity bar."""
import numpy as np
import pytest

from gms_liberi_b200 import liberi
from gms_liberi_b200 import molecules as M
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_F = 1e-10       # against the oracle
TOL_SAME = 1e-11    # batched vs single build: summation order of atomics only


def _mols():
    out = []
    for name in ("h2o_like", "ethane", "random_6", "random_9"):
        if name == "h2o_like":
            b, nocc = M.h2o_like(), 5
        elif name == "ethane":
            b, nocc = M.ethane(), 9
        else:
            b = M.random_molecule(int(name.split("_")[1]), seed=11)
            nocc = M.nocc_of(b)
        b["schwrz"] = oracle.schwarz(b)
        out.append((b, nocc))
    return out


def _setup(mols):
    hs = []
    for b, _ in mols:
        h = liberi.liberi_create()
        liberi.setup_from_basis(h, b)
        hs.append(h)
    return hs


def _device_buffers(mols, seed):
    import torch
    Ds, Fs = [], []
    for i, (b, nocc) in enumerate(mols):
        D = M.density(b["num_bas"], nocc, seed=seed + i)
        Ds.append(torch.tensor(D, dtype=torch.float64, device="cuda"))
        Fs.append(torch.full_like(Ds[-1], np.nan))  # the batch must zero F itself
    torch.cuda.synchronize()
    return Ds, Fs


def test_batch_equals_single_builds_and_oracle():
    mols = _mols()
    hs = _setup(mols)
    Ds, Fs = _device_buffers(mols, seed=3)
    singles = [liberi.fock(h, D.cpu().numpy()) for h, D in zip(hs, Ds)]
    bt = liberi.Batch(hs)
    bt.bind([d.data_ptr() for d in Ds], [f.data_ptr() for f in Fs])
    bt.fock_build()
    bt.synchronize()
    for (b, _), D, F, Fs1 in zip(mols, Ds, Fs, singles):
        Fb = F.cpu().numpy()
        assert np.abs(Fb - Fs1).max() <= TOL_SAME
        assert np.abs(Fb - oracle.fock_build(b, D.cpu().numpy())).max() <= TOL_F
    bt.destroy()
    for h in hs:
        liberi.liberi_destroy(h)


def test_batch_graph_replay_tracks_density():
    import torch
    mols = _mols()
    hs = _setup(mols)
    Ds, Fs = _device_buffers(mols, seed=7)
    bt = liberi.Batch(hs)
    bt.bind([d.data_ptr() for d in Ds], [f.data_ptr() for f in Fs])
    bt.capture()
    rng = np.random.default_rng(0)
    for it in range(3):  # SCF-style: D perturbed in place, the same graph replayed
        for D in Ds:
            D.add_(torch.tensor(1e-3 * rng.standard_normal(D.numel()), device="cuda"))
        torch.cuda.synchronize()
        bt.launch()
        bt.synchronize()
        for h, D, F in zip(hs, Ds, Fs):
            ref = liberi.fock(h, D.cpu().numpy())
            assert np.abs(F.cpu().numpy() - ref).max() <= TOL_SAME, it
    bt.destroy()
    for h in hs:
        liberi.liberi_destroy(h)


def test_autotune_keeps_results():
    import torch
    mols = _mols()
    hs = _setup(mols)
    Ds, Fs = _device_buffers(mols, seed=9)
    before = [liberi.fock(h, D.cpu().numpy()) for h, D in zip(hs, Ds)]
    # single handle
    chunks = liberi.autotune(hs[1], reps=1)
    assert set(chunks.tolist()) <= {0, 128, 256, 512, 1024, 2048}
    after = liberi.fock(hs[1], Ds[1].cpu().numpy())
    assert np.abs(after - before[1]).max() <= TOL_SAME
    # batch, captured first: the tuner re-captures with the tuned task lists
    bt = liberi.Batch(hs)
    bt.bind([d.data_ptr() for d in Ds], [f.data_ptr() for f in Fs])
    bt.capture()
    bchunks = bt.autotune(reps=1)
    assert set(bchunks.tolist()) <= {0, 128, 256, 512, 1024, 2048}
    for F in Fs:
        F.fill_(np.nan)
    torch.cuda.synchronize()
    bt.launch()
    bt.synchronize()
    for F, ref in zip(Fs, before):
        assert np.abs(F.cpu().numpy() - ref).max() <= TOL_SAME
    bt.destroy()
    for h in hs:
        liberi.liberi_destroy(h)


def test_batch_rejects_unusable_handles():
    mols = _mols()[:2]
    hs = _setup(mols)
    idle = liberi.liberi_create()
    with pytest.raises(liberi.LiberiError) as e:
        liberi.Batch([hs[0], idle])
    assert e.value.code == -2
    hs[1].set_option("precision", 1)
    with pytest.raises(liberi.LiberiError) as e:
        liberi.Batch(hs)
    assert e.value.code == -1
    bt = liberi.Batch([hs[0]])
    with pytest.raises(liberi.LiberiError):  # not bound yet
        bt.fock_build()
    with pytest.raises(liberi.LiberiError):  # nothing captured
        bt.launch()
    bt.destroy()
    for h in hs + [idle]:
        liberi.liberi_destroy(h)


def test_mixed_precision_batch_matches_single_mixed_builds():
    # the FP32/FP64 split of every molecule at its own max|D|, made on the
    # device inside the captured graph each iteration
    import torch
    mols = _mols()
    hs = []
    for b, _ in mols:
        h = liberi.liberi_create()
        h.set_option("precision", 1)
        h.set_option("fp32_cut", 1e-7)
        liberi.setup_from_basis(h, b)
        hs.append(h)
    Ds, Fs = _device_buffers(mols, seed=21)
    bt = liberi.Batch(hs)
    bt.bind([d.data_ptr() for d in Ds], [f.data_ptr() for f in Fs])
    bt.capture()
    rng = np.random.default_rng(3)
    for it in range(2):
        for D in Ds:
            D.mul_(1.0 + 0.1 * it).add_(torch.tensor(1e-3 * rng.standard_normal(D.numel()), device="cuda"))
        torch.cuda.synchronize()
        bt.launch()
        bt.synchronize()
        for (b, _), h, D, F in zip(mols, hs, Ds, Fs):
            Dh = D.cpu().numpy()
            alone = liberi.fock(h, Dh)
            assert np.abs(F.cpu().numpy() - alone).max() <= TOL_SAME, it
            # and within the mixed-precision bound of the FP64 oracle
            assert np.abs(F.cpu().numpy() - oracle.fock_build(b, Dh)).max() <= 1e-5
    bt.destroy()
    for h in hs:
        liberi.liberi_destroy(h)
