"""rmd_render_noalloc against rmd_render.

The allocation-free entry point serves callers that cannot allocate device
memory at render time (their host owns all GPU memory, or they run a loop
that must not allocate); it keeps its path state in a fixed array inside the
library and writes into a film the caller already owns.  This test gives it
a film allocated beforehand (here by torch, standing in for the caller's own
allocator), renders two samples with two calls in a row, and compares each
with the regular entry point's rendering of the same sample, with the parity
tolerance of the other GPU tests.  The file sorts last so that a run that
stops at the first failure has run every other test before it.
"""
import numpy as np
import pytest

from raymond_b200 import api, scenes
from raymond_b200._abi import SceneDesc

pytestmark = pytest.mark.gpu

REL, ABS, MIN_MATCH = 1e-3, 1e-6, 0.999


def test_noalloc_matches_regular_render(gpu_ctx):
    import torch

    W = H = 96
    desc = SceneDesc(scenes.cornell(seed=1, envmap_exponent=6))
    scene = api.Scene(gpu_ctx, desc)
    regular = api.Renderer(scene, W, H)
    films = [torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for s, film in enumerate(films):  # two calls in a row share the library's scratch array
        api.render_noalloc(scene, desc.scene["camera"], W, H, film.data_ptr(), spp=1, first_sample=s, max_depth=8)
    torch.cuda.synchronize()
    for s, film in enumerate(films):
        regular.reset()
        regular.render(spp=1, max_depth=8, first_sample=s)
        ref = regular.film().astype(np.float64)
        got = film.cpu().numpy()[..., :3].astype(np.float64)
        ok = np.abs(got - ref) <= REL * np.abs(ref) + ABS
        assert ok.all(axis=-1).mean() >= MIN_MATCH, s
        assert np.abs(got).sum() > 0


def test_noalloc_small_pool_allocates_nothing(gpu_ctx):
    """A pool of 1,024 paths carved from the array drains 32,768 paths in many
    regeneration rounds and matches rmd_render; after a first call, a second
    call leaves the device's free memory unchanged."""
    import torch

    W = H = 128
    desc = SceneDesc(scenes.cornell(seed=1, envmap_exponent=6))
    scene = api.Scene(gpu_ctx, desc)
    regular = api.Renderer(scene, W, H)
    regular.render(spp=2, max_depth=8, first_sample=0)
    ref = regular.film().astype(np.float64)
    films = [torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    api.render_noalloc(scene, desc.scene["camera"], W, H, films[0].data_ptr(), spp=2, first_sample=0,
                       max_depth=8, pool_size=1024)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    api.render_noalloc(scene, desc.scene["camera"], W, H, films[1].data_ptr(), spp=2, first_sample=0,
                       max_depth=8, pool_size=1024)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    for film in films:
        f = film.cpu().numpy()
        got = f[..., :3].astype(np.float64)
        ok = np.abs(got - ref) <= REL * np.abs(ref) + ABS
        assert ok.all(axis=-1).mean() >= MIN_MATCH
        assert np.all(f[..., 3] == 2)  # every pixel received both of its paths


def test_noalloc_rejects_oversized_pool(gpu_ctx):
    import torch

    desc = SceneDesc(scenes.cornell(seed=1, envmap_exponent=2))
    scene = api.Scene(gpu_ctx, desc)
    film = torch.zeros((8, 8, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(api.RmdError, match="RMD_NOALLOC_MAX_PATHS"):
        api.render_noalloc(scene, desc.scene["camera"], 8, 8, film.data_ptr(), spp=1, first_sample=0,
                           pool_size=32768 + 1)
