"""Replica sharding over processes, one per GPU.

Replicas are independent: replica r of a replay depends only on (seed, r,
node, step).  A rank that runs replicas [offset, offset + count) with
`replica_offset=offset` therefore produces exactly the slice of the
unsharded run, and the whole run is the concatenation of the ranks'
counts along the replica axis.  No data crosses between ranks during a
replay; the only exchange is the final gather of counts.

    import torch.distributed as dist
    dist.init_process_group("nccl")              # or "gloo"
    counts = run_sharded(graph, n_replicas=4096, iterations=336, ...)
"""
import numpy as np

__all__ = ["shard", "gather_counts", "run_sharded"]

ALIGN = 32  # replicas per random-stream word


def shard(n_replicas, world, rank):
    """(offset, count) of `rank`'s replicas: whole 32-replica words, split
    as evenly as possible (later ranks may hold fewer, or none)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    words = (n_replicas + ALIGN - 1) // ALIGN
    base, extra = divmod(words, world)
    w0 = rank * base + min(rank, extra)
    w1 = w0 + base + (1 if rank < extra else 0)
    off = min(w0 * ALIGN, n_replicas)
    return off, max(0, min(w1 * ALIGN, n_replicas) - off)


def gather_counts(local, n_replicas, group=None):
    """All-gathers every rank's counts (T+1, [networks,] count, 4) into the
    full (T+1, [networks,] n_replicas, 4) array on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    counts = [shard(n_replicas, world, r)[1] for r in range(world)]
    width = max(counts)
    local = np.asarray(local, np.int32)
    buf = np.zeros(local.shape[:-2] + (width, 4), np.int32)
    buf[..., :local.shape[-2], :] = local
    t = torch.from_numpy(buf)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    return np.concatenate([o.cpu().numpy()[..., :counts[r], :] for r, o in enumerate(outs)], axis=-2)


def run_sharded(graph, n_replicas, group=None, networks=None, **kw):
    """Runs this rank's replicas of an n_replicas replay on its GPU and
    returns the counts of all ranks (keyword arguments as Simulation; a
    beta_per_replica array covers all n_replicas and is sliced here)."""
    import torch.distributed as dist

    from . import Simulation
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    off, cnt = shard(n_replicas, world, rank)
    if kw.get("beta_per_replica") is not None:
        kw["beta_per_replica"] = np.asarray(kw["beta_per_replica"], np.float32)[off:off + cnt]
    steps = kw.get("iterations", kw.get("n_steps", 42))
    if cnt > 0:
        sim = Simulation(graph, networks=networks, M=cnt, replica_offset=off, **kw)
        local = sim.run()
        sim.close()
    else:
        shape = (steps + 1,) + ((len(networks) - 1,) if networks is not None else ()) + (0, 4)
        local = np.zeros(shape, np.int32)
    return gather_counts(local, n_replicas, group)
