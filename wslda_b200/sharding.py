"""State sharding of a run over several GPUs (one process and one context per GPU).

The quasiparticle states are independent between density evaluations, so a run of nwf states
splits into contiguous blocks, one per rank, exactly as the reference distributes them
(getnwfip, hpc-engine/pca_utils.c:660-664: nwf // np each, one more for the first nwf % np
ranks).  Each density reduction is then summed over ranks (the library's density exchange:
NCCL on the context stream, or a host hook), after which every rank holds the full densities
and computes the same potentials.
"""
import numpy as np


def shard_range(nwf, world, rank):
    """(offset, count) of this rank's block of states"""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(int(nwf), int(world))
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


def shard_rows(states, nwf, numel, world, rank):
    """this rank's states from the full [u_0..u_{nwf-1}, v_0..v_{nwf-1}] array (complex)"""
    off, cnt = shard_range(nwf, world, rank)
    y = np.asarray(states).reshape(2, nwf, numel)
    return np.ascontiguousarray(y[:, off:off + cnt, :]).reshape(-1)


def shard_vector(v, nwf, world, rank):
    """this rank's entries of a per-state array (occupations, k_perp, degeneracies)"""
    off, cnt = shard_range(nwf, world, rank)
    return None if v is None else np.ascontiguousarray(np.asarray(v)[off:off + cnt])


def gather_rows(shards, numel):
    """inverse of shard_rows: the rank blocks (in rank order) back into one state array"""
    us = [np.asarray(s).reshape(2, -1, numel) for s in shards]
    return np.concatenate([np.concatenate([s[0] for s in us]), np.concatenate([s[1] for s in us])]).reshape(-1)


def attach_nccl(run, rank, world, group=None):
    """give a TDRun an NCCL communicator over the ranks of torch.distributed: rank 0 makes the
    unique id, the process group carries it to the others"""
    import torch.distributed as dist
    box = [run.nccl_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    run.attach_nccl(box[0], world, rank)
