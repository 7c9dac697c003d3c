"""Multi-rank Fock builds: one process per GPU, torch.distributed for the
plumbing.

Every rank sets up its handle with (my_rank, num_procs); the engine then
evaluates either exactly the quartets the reference assigns that rank (the
per-kernel tile/chunk split of src/rhf/rot_axis/int0000.F90:76-91 and
int0001.F90:89-104, option rank_split 0) or a contiguous slice of every
class's work of equal primitive-quartet cost (rank_split 1), and returns a
partial packed F; the partials sum to the same F.  The caller's reduction
(GAMESS: DDI_GSUMF, liberi_interface.F90:13-15) is one all-reduce (sum) of the
packed F over NCCL.  There is no other data exchange: D is replicated.
"""
import torch
import torch.distributed as dist


def rank_and_world(group=None):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def reduced_fock(build_partial, group=None):
    """Sum of every rank's partial F.  `build_partial(rank, world)` returns
    this rank's packed partial F as a tensor (on the GPU for NCCL); the sum
    replaces it in place and is returned on every rank."""
    rank, world = rank_and_world(group)
    F = build_partial(rank, world)
    if world > 1:
        dist.all_reduce(F, op=dist.ReduceOp.SUM, group=group)
    return F


def max_over_ranks(x, device=None, group=None):
    """Maximum of a per-rank scalar (timings are reported as the slowest rank)."""
    _, world = rank_and_world(group)
    if world == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
