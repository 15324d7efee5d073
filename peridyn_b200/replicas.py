"""Host logic of the multi-GPU runs: one process per GPU, each advancing
independent specimens or serving its own share of a job stream.  The data
path has no collective (specimens do not interact); the only cross-rank
steps are the barrier before a timed region and the reductions of its
results (max of the elapsed times, sum of the work)."""
import os


def rank_info():
    """(rank, world_size, local_rank) from the torch.distributed launcher's
    environment (1 process when unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_by_footprint(sizes, world):
    """Deal items (e.g. jobs by particle count) to ``world`` ranks, largest
    first onto the least-loaded rank (ties to the lower rank).  Returns one
    ascending index list per rank; deterministic, so every rank computes the
    same assignment without communicating."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def reduce_timing(elapsed_s, work, dist=None, device="cpu"):
    """Whole-job figures of a timed region: the slowest rank's elapsed time
    and the work summed over ranks (every rank must call this)."""
    if dist is None:
        return float(elapsed_s), float(work)
    import torch

    t = torch.tensor([float(elapsed_s)], dtype=torch.float64, device=device)
    w = torch.tensor([float(work)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
