"""The multi-rank path on the CPU: two gloo ranks each build the partial F the
reference's rank split assigns them (the oracle stands in for the device
engine, whose per-rank partials are parity-tested against the same oracle
partials on the GPU), and the all-reduce of gms_liberi_b200.ranks sums them
to the full single-rank F; timings reduce to the slowest rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gms_liberi_b200 import molecules as M


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gms_liberi_b200 import ranks
        from oracle import oracle
        b = M.ethane()
        b["schwrz"] = oracle.schwarz(b)
        D = M.density(b["num_bas"], 9, seed=3)

        def partial(r, n):
            return torch.from_numpy(oracle.fock_build(b, D, schwarz_cut=1e-10, my_rank=r, num_procs=n))

        F = ranks.reduced_fock(partial)
        slow = ranks.max_over_ranks(10.0 * (rank + 1))
        mine = partial(rank, world).numpy()
        np.save(os.path.join(out_dir, "F_%d.npy" % rank), F.numpy())
        np.save(os.path.join(out_dir, "P_%d.npy" % rank), mine)
        np.save(os.path.join(out_dir, "T_%d.npy" % rank), np.array([slow]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_partials_sum_to_full_fock(world, tmp_path):
    from oracle import oracle
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    b = M.ethane()
    b["schwrz"] = oracle.schwarz(b)
    D = M.density(b["num_bas"], 9, seed=3)
    full = oracle.fock_build(b, D, schwarz_cut=1e-10)
    parts = [np.load(tmp_path / ("P_%d.npy" % r)) for r in range(world)]
    for r in range(world):
        F = np.load(tmp_path / ("F_%d.npy" % r))
        assert np.abs(F - full).max() <= 1e-12          # every rank holds the sum
        assert float(np.load(tmp_path / ("T_%d.npy" % r))[0]) == 10.0 * world
    # the split is a partition: no rank's share is empty, none is the whole
    for p in parts:
        assert 0 < np.abs(p).max() and np.abs(p - full).max() > 1e-6


def test_single_process_is_identity():
    from gms_liberi_b200 import ranks
    F = ranks.reduced_fock(lambda r, n: torch.arange(4, dtype=torch.float64) * (n - r))
    assert F.tolist() == [0.0, 1.0, 2.0, 3.0]
    assert ranks.max_over_ranks(3.5) == 3.5
