"""Multi-GPU plumbing: one process per GPU, paths independent, so work is
sharded without any exchange on the data path.

* `sample_range`: rank r of n renders samples [(r + n k) spp, ... + spp) of
  step k of one image (weak scaling: every rank adds its own samples).
* `shard_views`: views (instances) of a batch dealt round-robin to ranks.
* `max_over_ranks` / `sum_over_ranks`: the host-side reductions of
  timings and counts (gloo on CPU, NCCL on GPUs).
* `gather_films`: the views' films brought to rank 0 (host gather).
* `reduce_film` / `combine_films`: one image whose samples were split over
  ranks, summed into rank 0's film: an NCCL reduce on the device films in
  place (gloo on host tensors).

The process group comes from torch.distributed (launched by torchrun, one
rank per GPU); without one, every helper acts as a world of one.
"""
from __future__ import annotations

import os
from typing import Any

import numpy as np


def rank_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def sample_range(rank: int, world: int, step: int, spp: int) -> tuple[int, int]:
    """First sample and count of this rank's share of step `step`."""
    first = (rank + world * step) * spp
    return first, spp


def shard_views(num_views: int, rank: int, world: int) -> list[int]:
    """The views this rank renders (round-robin, so sizes that grow with the
    index spread over ranks)."""
    return list(range(rank, num_views, world))


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover
        return None
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(values: list[float]) -> list[float]:
    dist = _dist()
    if dist is None:
        return list(values)
    import torch

    t = torch.tensor(values, dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().tolist()


def sum_over_ranks(values: list[float]) -> list[float]:
    dist = _dist()
    if dist is None:
        return list(values)
    import torch

    t = torch.tensor(values, dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().tolist()


def gather_films(films: dict[int, np.ndarray]) -> dict[int, np.ndarray] | None:
    """Every rank's {view: film}; rank 0 receives the union, others None."""
    dist = _dist()
    if dist is None:
        return dict(films)
    out: list[Any] = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(films, out, dst=0)
    if dist.get_rank() != 0:
        return None
    merged: dict[int, np.ndarray] = {}
    for part in out:
        merged.update(part)
    return merged


def reduce_film(film):
    """Sum a film tensor over ranks into rank 0's, in place.  The other ranks'
    tensors hold unspecified values afterwards (a reduce may keep partial sums
    there).  A CUDA tensor under NCCL, a CPU tensor under gloo.  Returns the
    tensor on rank 0, None elsewhere."""
    dist = _dist()
    if dist is None:
        return film
    dist.reduce(film, dst=0, op=dist.ReduceOp.SUM)
    return film if dist.get_rank() == 0 else None


def combine_films(renderer) -> int:
    """The frame of all ranks: every rank's renderer holds its own disjoint
    samples of one image; their films are summed into rank 0's renderer, whose
    sample count becomes the total (the other ranks' films are left unspecified).  `renderer.film_tensor()` aliases the
    film: on GPUs a zero-copy CUDA view of the library's buffer, reduced by
    NCCL in place.  Returns the total sample count."""
    total = int(sum_over_ranks([float(renderer.samples())])[0])
    dist = _dist()
    if dist is None:
        return total
    film = renderer.film_tensor()
    if film.is_cuda:
        import torch

        torch.cuda.synchronize()  # the renderer's stream has finished before the collective reads
        reduce_film(film)
        torch.cuda.synchronize()  # the sum is in place before the library's stream reads the film again
    else:
        reduce_film(film)
    if dist.get_rank() == 0:
        renderer.set_samples(total)
    return total
