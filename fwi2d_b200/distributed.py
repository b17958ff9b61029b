"""Shot sharding over processes (one process per GPU).

The reference distributes shots round-robin over MPI ranks and sums the
gradients with MPI_Allreduce (src/cpp/we_op.cpp:1136-1190,
src/include/optimization.hpp:609-618, 898-912).  Here each rank takes a
cost-balanced share of the shots (cost = grid cells x time samples) and the
model gradient and misfit are summed with one torch.distributed all-reduce
(NCCL on GPUs, gloo in the CPU tests).  The propagation itself needs no
collective: shots are independent.
"""


def shot_cost(shot, nz):
    return int(shot["nx"]) * int(nz) * int(shot["nt"])


def shard_shots(shots, rank, world, nz=1):
    """Indices of the shots rank `rank` computes: longest-processing-time
    assignment (largest cost first to the least-loaded rank, ties to the lower
    rank), returned in increasing shot order.  Deterministic."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    order = sorted(range(len(shots)), key=lambda i: (-shot_cost(shots[i], nz), i))
    load = [0] * world
    owner = [0] * len(shots)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += shot_cost(shots[i], nz)
    return [i for i in range(len(shots)) if owner[i] == rank]


def allreduce_sum(tensor, group=None):
    """In-place sum over ranks (gradient, misfit)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor
