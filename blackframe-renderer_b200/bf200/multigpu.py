"""Multi-GPU frames: one process per GPU, each rendering a disjoint sample range of the same
frame into its own film, and one all-reduce (sum) of the films.

Every random number of a path is indexed by (seed, pixel, sample, dimension), so a path's result
does not depend on which GPU traced it; the sum of the per-GPU films equals the film of the whole
sample range up to floating-point summation order. The film reduce is the path's only exchange
step (NCCL over NVLink on B200s; any torch.distributed backend works).
"""


def rank_sample_range(step, rank, world, samples_per_pixel):
    """First and end sample index of `rank` in frame step `step`: rank r of N renders the
    samples [(step * N + r) * spp, (step * N + r + 1) * spp) of every pixel."""
    first = (step * world + rank) * samples_per_pixel
    return first, first + samples_per_pixel


def batch_shard(job_paths, rank, world):
    """The jobs of a multi-scene batch that `rank` of `world` renders: whole jobs, no exchange.
    Jobs go largest first to the rank with the fewest paths so far (ties to the lowest rank), so
    uneven jobs balance; every job goes to exactly one rank. Returns job indices in ascending order."""
    order = sorted(range(len(job_paths)), key=lambda j: (-job_paths[j], j))
    load = [0] * world
    owner = [0] * len(job_paths)
    for j in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[j] = r
        load[r] += job_paths[j]
    return [j for j in range(len(job_paths)) if owner[j] == rank]


def reduce_film(sums, counts=None):
    """Sums the per-rank films in place on every rank (torch tensors on the process group's
    device). Sample counts are summed as well when given."""
    import torch.distributed as dist

    dist.all_reduce(sums)
    if counts is not None:
        dist.all_reduce(counts)
