"""Per-sample parity on the workloads the bench measures, at their full sizes.

The same criterion as tests/test_parity_gpu.py: same seed and PCG32 stream per
path; a pixel matches when every channel satisfies
|gpu - cpu| <= 1e-3 |cpu| + 1e-6, and at least 99.9 % of pixels must match.

- Spheres on terrain (the throughput benchmark): the full 851,968-triangle
  scene, 1920 x 1080, depth 12, three single samples, every pixel.
- Glossy room (the guided benchmark's scene, plain tracer): 197,490 triangles,
  roughness down to 0.02, lit by a constant environment through one window;
  1280 x 720, depth 16, every pixel, 16 samples accumulated (one sample lights
  only ~0.1 % of the pixels); the bar also on the lit pixels alone (>= 99 %).
- 4 x 4 glossy rooms (the guided batch's scene): 3,949,856 triangles,
  metallic Bernoulli(0.5), roughness down to 0.01, 64 emitters of radiance
  500; all 8 views at 3840 x 2160, depth 20, rendered as one batch; the
  oracle checks every 7th pixel of each view (1.18 M pixels per view), with
  the bar set by the scene's own sensitivity to rounding (the test's
  docstring).
"""
import numpy as np
import pytest

import oracle_ctypes as O
from raymond_b200 import api, scenes
from raymond_b200._abi import SceneDesc

pytestmark = pytest.mark.gpu

REL, ABS, MIN_MATCH = 1e-3, 1e-6, 0.999


def match_fraction(gpu, cpu, pixels=None):
    g = gpu.reshape(-1, 3).astype(np.float64)
    c = cpu.reshape(-1, 3)
    if pixels is not None:
        g, c = g[pixels], c[pixels]
    ok = np.abs(g - c) <= REL * np.abs(c) + ABS
    return float(ok.all(axis=-1).mean())


def test_spheres_terrain_full_frame(gpu_ctx):
    desc = SceneDesc(scenes.spheres_terrain(seed=1))
    scene = api.Scene(gpu_ctx, desc)
    assert scene.info()["triangles"] == 851968
    orc = O.OracleScene(desc)
    W, H, depth = 1920, 1080, 12
    r = api.Renderer(scene, W, H)
    for s in (0, 1, 2):
        r.reset()
        r.render(spp=1, max_depth=depth, first_sample=s)
        cpu, st = orc.render(W, H, 1, depth, first_sample=s)
        assert match_fraction(r.film(), cpu) >= MIN_MATCH, s
        g = r.stats()
        assert abs(g["segments"] - st["segments"]) <= 1e-3 * st["segments"]


def test_glossy_room_full_frame(gpu_ctx):
    """Few paths find the window (about 0.1 % of the pixels receive light in
    one sample), so 16 samples are accumulated, the same 16 on both sides: a
    pixel matches only if its 16 paths do.  The bar also holds on the lit
    pixels alone, and there must be enough of them."""
    desc = SceneDesc(scenes.glossy_room(seed=1))
    scene = api.Scene(gpu_ctx, desc)
    orc = O.OracleScene(desc)
    W, H, depth, spp = 1280, 720, 16, 16
    r = api.Renderer(scene, W, H)
    r.render(spp=spp, max_depth=depth, first_sample=0)
    cpu, _ = orc.render(W, H, spp, depth, first_sample=0)
    gpu = r.film()
    assert match_fraction(gpu, cpu) >= MIN_MATCH
    lit = np.flatnonzero(cpu.reshape(-1, 3).sum(axis=-1) > 0)
    assert len(lit) >= 5000, len(lit)
    assert match_fraction(gpu, cpu, lit) >= 0.99


def test_glossy_rooms_grid_all_views(gpu_ctx):
    """The 4 x 4 rooms amplify rounding.  Their metallic faces reach
    roughness 0.01 (GGX alpha 1e-4), where the microfacet distribution near its
    peak is computed from cos^2(theta) (alpha^2 - 1) + 1, a difference FP32
    cannot resolve, and the radiance-500 emitters seen through those lobes
    light most of the lit pixels; so one ulp anywhere on a path can move its
    sample by more than 1e-3.  The oracle built with contracted multiply-adds
    (oracle_ctypes.LIB_FMA), the same code whose results move by about an ulp,
    differs from the oracle on 0.15-0.55 % of these pixels (5-16 % of the lit
    ones), so the fixed 99.9 % bar cannot hold for any second implementation.
    The bar is that rounding floor: over all views the GPU misses the
    per-sample criterion on at most 1.25 x as many pixels as the contracted
    oracle does (all pixels, and the lit ones), and on at most 2 x as many in
    each view (or passes the fixed bars outright)."""
    if not O.fma_available():
        pytest.skip("the contracted oracle needs FMA instructions on the host CPU")
    desc = SceneDesc(scenes.glossy_rooms_grid(seed=1))
    cams = scenes.grid_views(8)
    W, H, depth = 3840, 2160, 20
    b = api.Batch(gpu_ctx, [desc], [{"scene": 0, "width": W, "height": H, "camera": c} for c in cams])
    b.render(spp=1, max_depth=depth, first_sample=0)
    orc, orc_fma = O.OracleScene(desc), O.OracleScene(desc, "fma")
    pixels = np.arange(0, W * H, 7, dtype=np.uint32)
    totals = np.zeros((2, 2))  # [gpu, contracted oracle] x [all, lit] mismatching pixels
    lit_total = 0
    for v, cam in enumerate(cams):
        orc.set_camera(cam)
        orc_fma.set_camera(cam)
        cpu, _ = orc.render(W, H, 1, depth, first_sample=0, pixels=pixels)
        ref, _ = orc_fma.render(W, H, 1, depth, first_sample=0, pixels=pixels)
        gpu = b.film(v)
        lit = pixels[cpu.reshape(-1, 3)[pixels].sum(axis=-1) > 0]
        assert len(lit) >= 0.005 * len(pixels), (v, len(lit))
        lit_total += len(lit)
        for k, (px, bar) in enumerate(((pixels, MIN_MATCH), (lit, 0.99))):
            miss_gpu = 1.0 - match_fraction(gpu, cpu, px)
            miss_ref = 1.0 - match_fraction(ref, cpu, px)
            print(f"view {v} {'lit' if k else 'all'}: gpu misses {miss_gpu:.5f}, contracted oracle {miss_ref:.5f}")
            assert miss_gpu <= max(1.0 - bar, 2.0 * miss_ref), (v, k, miss_gpu, miss_ref)
            totals[:, k] += np.array([miss_gpu, miss_ref]) * len(px)
    b.close()
    for k in range(2):
        assert totals[0, k] <= 1.25 * totals[1, k] or totals[0, k] <= (1.0 - MIN_MATCH) * len(pixels) * len(cams), \
            (k, totals)
