"""The multi-GPU host logic on CPU: two gloo ranks (one per would-be GPU)
check that sample ranges and view shards are disjoint and complete, that the
timing reduction takes the maximum over ranks, that the films of all ranks'
views reach rank 0, and that the films of one image split over the ranks'
sample ranges sum into rank 0's film with the total sample count."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

from raymond_b200 import multi


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _FakeRenderer:
    """Stands in for api.Renderer on the CPU: rank r's film holds its own 2
    samples of a 4 x 5 image (RGB = radiance, A = path count)."""

    def __init__(self, rank):
        g = np.random.default_rng(100 + rank)
        self.film = torch.from_numpy(np.concatenate([g.uniform(0, 1, (4, 5, 3)), np.full((4, 5, 1), 2.0)],
                                                    axis=-1).astype(np.float32))
        self.samples_set = None

    def samples(self):
        return 2

    def film_tensor(self):
        return self.film

    def set_samples(self, n):
        self.samples_set = n


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = multi.rank_info()
        samples = [multi.sample_range(r, w, k, 4) for k in range(3)]
        views = multi.shard_views(7, r, w)
        mx = multi.max_over_ranks([float(r + 1), 10.0 - r])
        tot = multi.sum_over_ranks([1.0])
        films = {v: np.full((2, 3, 3), v, np.float32) for v in views}
        merged = multi.gather_films(films)
        # one image split over the ranks' sample ranges: films summed into rank 0's
        fake = _FakeRenderer(r)
        total = multi.combine_films(fake)
        q.put((r, samples, views, mx, tot, None if merged is None else sorted(merged),
               total, fake.film.numpy().copy(), fake.samples_set))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    sample_sets = [set(range(f, f + n)) for _, samples, *_ in results for f, n in samples]
    allsamples = set().union(*sample_sets)
    assert sum(len(s) for s in sample_sets) == len(allsamples) == world * 3 * 4  # disjoint, no gaps
    assert allsamples == set(range(world * 3 * 4))
    views = [v for _, _, vs, *_ in results for v in vs]
    assert sorted(views) == list(range(7))
    for _, _, _, mx, tot, *_ in results:
        assert mx == [2.0, 10.0] and tot == [2.0]
    assert results[0][5] == list(range(7)) and results[1][5] is None
    # the summed frame on rank 0: both ranks' radiance, 4 paths per pixel, 4 samples
    expect = sum(_FakeRenderer(r).film.numpy() for r in range(world))
    assert results[0][6] == results[1][6] == 4
    np.testing.assert_allclose(results[0][7], expect, rtol=1e-6)
    assert np.all(results[0][7][..., 3] == 4.0) and results[0][8] == 4
    assert results[1][8] is None


def test_world_of_one_without_process_group():
    assert multi.max_over_ranks([3.0]) == [3.0]
    assert multi.shard_views(3, 0, 1) == [0, 1, 2]
    assert sorted(multi.gather_films({0: np.zeros(1)})) == [0]
