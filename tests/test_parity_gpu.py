"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Criterion for images: same seed, same PRNG stream per path; per-sample
radiance of a pixel matches when every channel satisfies
|gpu - cpu| <= 1e-3 * |cpu| + 1e-6, and at least 99.9 % of pixels must match.
"""
import numpy as np
import pytest

import oracle_ctypes as O
from raymond_b200 import api, scenes
from raymond_b200._abi import (RNG_PCG32, RNG_TEA, SAMPLING_BSDF, SAMPLING_MIS, SAMPLING_NEE, TONEMAP_ACES,
                               TONEMAP_HABLE, TONEMAP_LINEAR, SceneDesc, default_uniforms)

pytestmark = pytest.mark.gpu

REL, ABS, MIN_MATCH = 1e-3, 1e-6, 0.999


def match_fraction(gpu, cpu):
    ok = np.abs(gpu.astype(np.float64) - cpu) <= REL * np.abs(cpu) + ABS
    return float(ok.all(axis=-1).mean())


@pytest.fixture(scope="module")
def cornell(gpu_ctx):
    desc = SceneDesc(scenes.cornell(seed=1, envmap_exponent=11))
    return desc, api.Scene(gpu_ctx, desc), O.OracleScene(desc)


def per_sample(desc, scene, orc, W, H, samples, depth, **kw):
    r = api.Renderer(scene, W, H)
    fracs = []
    for s in samples:
        r.reset()
        r.render(spp=1, max_depth=depth, first_sample=s, **kw)
        gpu = r.film()
        cpu, stats = orc.render(W, H, 1, depth, first_sample=s, sampling_mode=kw.get("sampling_mode", SAMPLING_MIS),
                                rng=kw.get("rng", RNG_PCG32), seed=kw.get("seed", 1))
        fracs.append(match_fraction(gpu, cpu))
    return fracs


def test_prng_bit_exact(built):
    for mode, a, b in [(RNG_PCG32, 1, 0), (RNG_PCG32, 1, 123456789012), (RNG_TEA, 1, 77), (RNG_TEA, 99, 4242)]:
        g = api.test_prng(mode, a, b, 257)
        c = O.prng(mode, a, b, 257)
        assert np.array_equal(g.view(np.uint32), c.view(np.uint32)), (mode, a, b)


def test_cornell_per_sample_pcg(cornell):
    """Config 1: 256x256, depth 8, PCG32 seed 1, all 16 samples one by one."""
    desc, scene, orc = cornell
    fr = per_sample(desc, scene, orc, 256, 256, range(16), 8)
    assert min(fr) >= MIN_MATCH, fr


def test_cornell_accumulated_16spp(cornell):
    desc, scene, orc = cornell
    r = api.Renderer(scene, 256, 256)
    r.render(spp=16, max_depth=8)
    gpu = r.film()
    cpu, st = orc.render(256, 256, 16, 8)
    assert match_fraction(gpu, cpu) >= MIN_MATCH
    s = r.stats()
    assert s["paths"] == 16 * 256 * 256
    # segments (closest-hit rays shaded) agree up to the paths that diverged
    assert abs(s["segments"] - st["segments"]) <= 1e-3 * st["segments"]
    # every path traces at least its camera ray; misses are rays but not segments
    assert s["rays"] >= s["segments"] and s["rays"] >= s["paths"]


@pytest.mark.parametrize("mode", [SAMPLING_BSDF, SAMPLING_NEE])
def test_cornell_sampling_modes(cornell, mode):
    desc, scene, orc = cornell
    fr = per_sample(desc, scene, orc, 96, 96, [0, 5], 8, sampling_mode=mode)
    assert min(fr) >= MIN_MATCH, fr


def test_cornell_tea_reference_rng(cornell):
    """The reference's TEA generator seeded per frame as generateRays does."""
    desc, scene, orc = cornell
    fr = per_sample(desc, scene, orc, 128, 128, [0, 3], 8, rng=RNG_TEA)
    assert min(fr) >= MIN_MATCH, fr


@pytest.fixture(scope="module")
def spheres(gpu_ctx):
    sc = scenes.spheres_terrain(seed=3, num_spheres=12, terrain_cells=64, envmap_exponent=6)
    desc = SceneDesc(sc)
    return desc, api.Scene(gpu_ctx, desc), O.OracleScene(desc)


def test_spheres_terrain_per_sample(spheres):
    """Config-2 shading graph (noise -> ramp -> mix -> Principled), sun + point lights, depth 12."""
    desc, scene, orc = spheres
    fr = per_sample(desc, scene, orc, 160, 90, [0, 1, 2], 12)
    assert min(fr) >= MIN_MATCH, fr


def test_trace_parity(spheres):
    desc, scene, orc = spheres
    rng = np.random.default_rng(7)
    n = 20000
    o = rng.uniform([0, 0, 0], [20, 8, 20], (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, np.full((n, 1), 1e-3), d, np.full((n, 1), 1e30)], 1).astype(np.float32)
    g, gi = scene.trace(rays)
    c, ci = orc.trace(rays)
    # both return the closest hit of an exhaustive search with the same
    # triangle test and tie-break, so every record is identical bit for bit
    assert (c[:, 0] > 0).mean() > 0.25
    np.testing.assert_array_equal(g.view(np.uint32), c.view(np.uint32))
    np.testing.assert_array_equal(gi, ci)
    ga, _ = scene.trace(rays, any_hit=True)
    ca, _ = orc.trace(rays, any_hit=True)
    np.testing.assert_array_equal(ga[:, 0], ca[:, 0])


def test_material_eval_parity(spheres):
    """One material's node graph + UberShader evaluate/sample on random inputs."""
    desc, scene, orc = spheres
    rng = np.random.default_rng(11)
    n = 4096
    rec = np.zeros((n, 28), np.float32)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    nrm = unit(n)
    rec[:, 0:3] = rng.uniform(0, 20, (n, 3))
    rec[:, 3:6] = nrm
    rec[:, 6:9] = nrm
    rec[:, 9:12] = rng.uniform(0, 1, (n, 3))
    rec[:, 12:15] = rng.uniform(0, 1, (n, 3))
    wo = unit(n)
    wo *= np.sign(np.sum(wo * nrm, 1, keepdims=True))
    rec[:, 15:18] = wo
    rec[:, 18:21] = unit(n)
    rec[:, 21:24] = rng.uniform(0, 1, (n, 3))
    rec[:, 24] = 1
    for m in [0, 5, 12]:
        g = scene.material_eval(m, rec)
        c = orc.material_eval(m, rec)
        close = np.isclose(g, c, rtol=1e-3, atol=1e-5) | (np.isnan(g) & np.isnan(c))
        assert close.all(axis=1).mean() > 0.999, m


def _pin_modules():
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "ref"))
    import pin_materials
    import ref_ctypes

    return pin_materials, ref_ctypes


def test_pin_materials_parity(gpu_ctx):
    """Every pinning material (the node set checked against the reference's own
    node library on the CPU, Mapping, Normal Map, Hue/Saturation,
    Bright/Contrast and Blackbody included) evaluated and sampled on the GPU
    against the oracle, with a tangent frame in the records."""
    pin, R = _pin_modules()
    desc = SceneDesc(pin.scene())
    scene = api.Scene(gpu_ctx, desc)
    orc = O.OracleScene(desc)
    rec = R.shading_records(4096, seed=123)
    for m, (name, _) in enumerate(pin.materials()):
        g = scene.material_eval(m, rec)
        c = orc.material_eval(m, rec)
        close = np.isclose(g, c, rtol=1e-3, atol=1e-5) | (np.isnan(g) & np.isnan(c))
        assert close.all(axis=1).mean() > 0.999, name


def test_next_node_set_render(gpu_ctx):
    """The Cornell box with its walls in the Mapping / Hue / Bright-Contrast /
    tangent Normal Map material and its boxes in the Blackbody / world Normal
    Map one: per-sample parity with the oracle (tangents from the UVs)."""
    pin, _ = _pin_modules()
    sc = scenes.cornell(seed=1, envmap_exponent=7)
    mats = dict(pin.materials())
    base = len(sc["materials"])
    sc["materials"] = sc["materials"] + [("nodes_a", mats["mapping_hue_normal_map"]),
                                         ("nodes_b", mats["blackbody_world_normal"])]
    for i, sh in enumerate(sc["shapes"][:-1]):  # all but the light
        sh["materials"] = np.full_like(sh["materials"], base + (0 if i < 5 else 1))
    desc = SceneDesc(sc)
    scene = api.Scene(gpu_ctx, desc)
    orc = O.OracleScene(desc)
    fr = per_sample(desc, scene, orc, 96, 96, range(4), 8)
    assert min(fr) >= MIN_MATCH, fr


def test_image_textures_render(gpu_ctx):
    """The Cornell box with its walls and boxes in the image-texture material
    (an sRGB byte image through a Mapping, a 16-bit single-channel image, a
    float environment image and a missing file) and the textures in the scene:
    per-sample parity with the oracle."""
    pin, _ = _pin_modules()
    sc = scenes.cornell(seed=1, envmap_exponent=7)
    mats = dict(pin.materials())
    base = len(sc["materials"])
    sc["materials"] = sc["materials"] + [("textured", mats["image_textures"])]
    sc["textures"] = pin.textures()
    for sh in sc["shapes"][:-1]:
        sh["materials"] = np.full_like(sh["materials"], base)
    desc = SceneDesc(sc)
    scene = api.Scene(gpu_ctx, desc)
    orc = O.OracleScene(desc)
    fr = per_sample(desc, scene, orc, 96, 96, range(4), 8)
    assert min(fr) >= MIN_MATCH, fr


def test_non_finite_samples_dropped_and_counted(gpu_ctx):
    """A material whose base colour is NaN (a Math node's power of -1 to 0.5):
    its light and BSDF samples are dropped, as the reference drops them, the
    film stays finite and the renderer counts them."""
    pin, _ = _pin_modules()
    sc = scenes.cornell(seed=1, envmap_exponent=4)
    nan_mat = {
        "Math": {"type": "MATH", "parameters": {"operation": "POWER", "use_clamp": False},
                 "inputs": {"Value": {"type": "VALUE", "value": -1.0}, "Value_001": {"type": "VALUE", "value": 0.5},
                            "Value_002": {"type": "VALUE", "value": 0.0}}},
        "Principled BSDF": {"type": "BSDF_PRINCIPLED",
                            "inputs": dict(pin.M.principled_inputs(),
                                           **{"Base Color": {"type": "RGBA", "links": [["Math", "Value"]]}}),
                            "parameters": {"distribution": "GGX", "subsurface_method": "RANDOM_WALK"}},
        "Material Output": {"type": "OUTPUT_MATERIAL", "parameters": {},
                            "inputs": {"Surface": {"type": "SHADER", "links": [["Principled BSDF", "BSDF"]]}}},
    }
    sc["materials"] = sc["materials"] + [("nan", nan_mat)]
    sc["shapes"][0]["materials"] = np.full_like(sc["shapes"][0]["materials"], len(sc["materials"]) - 1)  # floor
    r = api.Renderer(api.Scene(gpu_ctx, SceneDesc(sc)), 64, 64)
    r.render(spp=4, max_depth=8)
    assert np.all(np.isfinite(r.film()))
    assert r.stats()["invalid_samples"] > 0
    plain = api.Renderer(api.Scene(gpu_ctx, SceneDesc(scenes.cornell(seed=1, envmap_exponent=4))), 64, 64)
    plain.render(spp=4, max_depth=8)
    assert plain.stats()["invalid_samples"] == 0


def _all_lights_scene():
    return scenes.cornell_all_lights(seed=4, envmap_exponent=7)


@pytest.mark.parametrize("mode", [SAMPLING_MIS, SAMPLING_NEE])
def test_all_light_types_per_sample(gpu_ctx, mode):
    desc = SceneDesc(_all_lights_scene())
    scene = api.Scene(gpu_ctx, desc)
    orc = O.OracleScene(desc)
    assert orc.info()["lights"] == 1 + 2 + 2 + 1 + 1 + 1
    fr = per_sample(desc, scene, orc, 96, 96, [0, 7], 6, sampling_mode=mode)
    assert min(fr) >= MIN_MATCH, fr


def test_fp64_film_matches_fp32(cornell):
    desc, scene, orc = cornell
    r = api.Renderer(scene, 64, 64)
    r.render(spp=4, max_depth=8, film_fp64=True)
    f64 = r.film64()
    cpu, _ = orc.render(64, 64, 4, 8, film_fp64=True)
    assert match_fraction(f64, cpu) >= MIN_MATCH


def test_autotune_keeps_parity(cornell):
    desc, scene, orc = cornell
    r = api.Renderer(scene, 128, 128, pool_size=1 << 16)
    res = r.autotune(spp=8, max_depth=8)
    assert res["shade_min_blocks"] in (1, 3, 4, 5, 6)
    assert res["pool_size"] >= 1 << 15 and res["ms_best"] <= res["ms_default"] * 1.0001
    assert r.samples() == 0  # the film was cleared
    for s in (0, 9):
        r.reset()
        r.render(spp=1, max_depth=8, first_sample=s)
        cpu, _ = orc.render(128, 128, 1, 8, first_sample=s)
        assert match_fraction(r.film(), cpu) >= MIN_MATCH


def test_set_tuning_keeps_parity(cornell):
    """Launch choices applied by hand (another process's autotune result)."""
    desc, scene, orc = cornell
    cpu, _ = orc.render(128, 128, 1, 8, first_sample=2)
    r = api.Renderer(scene, 128, 128)
    r.set_tuning({"shade_min_blocks": 3, "trace_blocks_per_sm": 4, "pool_size": 4096})
    r.render(spp=1, max_depth=8, first_sample=2)
    assert r.stats()["pool_size"] == 4096
    assert match_fraction(r.film(), cpu) >= MIN_MATCH
    with pytest.raises(api.RmdError):
        r.set_tuning({"shade_min_blocks": 0, "trace_blocks_per_sm": 4, "pool_size": 0})


@pytest.mark.parametrize("tonemapping", [TONEMAP_LINEAR, TONEMAP_HABLE, TONEMAP_ACES])
def test_film_tonemap(cornell, tonemapping):
    """normalizeImage on the GPU (rmd_film_read and rmd_film_normalize with the
    reference's Uniforms) against the oracle's restatement, which is pinned bit
    for bit to the reference's kernel; the GPU may fuse multiply-adds, so the
    bar is 1e-5 relative + 1e-6 absolute (the Hable curve subtracts nearly
    equal terms near black)."""
    desc, scene, orc = cornell
    r = api.Renderer(scene, 64, 64)
    r.render(spp=4, max_depth=8)
    raw = r.film()
    got = r.film(normalize=True, tonemapping=tonemapping, exposure=1.7)
    ref = O.normalize_image(raw, 1.7, True, 3, tonemapping)
    np.testing.assert_allclose(got, ref[..., :3], rtol=1e-5, atol=1e-6)
    for accumulate in (1, 0):
        u = default_uniforms(exposure=0.8, tonemapping=tonemapping, frame_index=3, accumulate=accumulate)
        got4 = r.film_normalize(u)
        ref4 = O.normalize_image(raw, 0.8, bool(accumulate), 3, tonemapping)
        np.testing.assert_allclose(got4, ref4, rtol=1e-5, atol=1e-6)


def test_render_frame_uniforms(cornell):
    """rmd_render_frame: frames driven by the reference's Uniforms equal the
    oracle's TEA frames (random seed k = sample k - 1); accumulate = 0 clears
    the film first."""
    desc, scene, orc = cornell
    W = H = 80
    r = api.Renderer(scene, W, H)
    for frame in range(3):
        r.render_frame(default_uniforms(frame_index=frame, random_seed=frame + 1, accumulate=1), max_depth=8)
    cpu, _ = orc.render(W, H, 3, 8, rng=RNG_TEA, first_sample=0)
    assert match_fraction(r.film(), cpu) >= MIN_MATCH
    r.render_frame(default_uniforms(random_seed=5, accumulate=0, sampling_mode=SAMPLING_NEE), max_depth=8)
    cpu, _ = orc.render(W, H, 1, 8, rng=RNG_TEA, first_sample=4, sampling_mode=SAMPLING_NEE)
    assert match_fraction(r.film(), cpu) >= MIN_MATCH
    with pytest.raises(api.RmdError):
        r.render_frame(default_uniforms(num_lens_surfaces=3))


def _sky_world(sky_type):
    params = {"sky_type": sky_type, "sun_elevation": 0.3, "sun_rotation": 2.0, "sun_disc": True, "sun_size": 0.08,
              "sun_intensity": 1.0, "altitude": 100.0, "air_density": 1.0, "dust_density": 1.5,
              "ozone_density": 1.0, "sun_direction": [0.3, -0.5, 0.4], "turbidity": 2.2, "ground_albedo": 0.3}
    return {
        "Sky Texture": {"type": "TEX_SKY", "inputs": {"Vector": {"type": "VECTOR", "value": [0.0, 0.0, 0.0]}},
                        "parameters": params},
        "Background": {"type": "BACKGROUND", "parameters": {},
                       "inputs": {"Color": {"type": "RGBA", "links": [["Sky Texture", "Color"]]},
                                  "Strength": {"type": "VALUE", "value": 0.05},
                                  "Weight": {"type": "VALUE", "value": 0.0}}},
        "World Output": {"type": "OUTPUT_WORLD", "parameters": {},
                         "inputs": {"Surface": {"type": "SHADER", "links": [["Background", "Background"]]},
                                    "Volume": {"type": "SHADER"}}},
    }


@pytest.mark.parametrize("sky_type", ["NISHITA", "HOSEK_WILKIE"])
def test_sky_world_per_sample(gpu_ctx, sky_type):
    """The Nishita sky node (its 512 x 512 texture generated on the device)
    lighting the all-lights room through its open front, the environment
    importance map built from it: per-sample parity with the oracle, whose
    sky model is pinned to the reference's own."""
    sc = scenes.cornell_all_lights(seed=4, envmap_exponent=7)
    sc["light_materials"][0] = ("world", _sky_world(sky_type))
    desc = SceneDesc(sc)
    scene = api.Scene(gpu_ctx, desc)
    orc = O.OracleScene(desc)
    fr = per_sample(desc, scene, orc, 96, 96, [0, 1], 8)
    assert min(fr) >= MIN_MATCH, fr
    r = api.Renderer(scene, 96, 96)
    r.render(spp=1, max_depth=8, first_sample=0)
    assert np.isfinite(r.film()).all() and r.film().sum() > 0


def test_film_device_view_and_sample_count(cornell):
    """rmd_film_device: a zero-copy torch view of the renderer's film equals the
    read-back film; a film summed into it (as the ranks' films are by the NCCL
    reduce) is what rmd_film_read returns, normalised by the sample count set
    with rmd_film_set_samples."""
    import torch

    desc, scene, orc = cornell
    a = api.Renderer(scene, 64, 48)
    b = api.Renderer(scene, 64, 48)
    a.render(spp=2, max_depth=8, first_sample=0)
    b.render(spp=2, max_depth=8, first_sample=2)
    ta, tb = a.film_tensor(), b.film_tensor()
    assert ta.shape == (48, 64, 4) and ta.is_cuda
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ta[..., :3].cpu().numpy(), a.film())
    assert torch.all(ta[..., 3] == 2)  # two paths per pixel
    ta += tb  # the sum a reduce over two ranks leaves in rank 0's film
    torch.cuda.synchronize()
    a.set_samples(4)
    assert a.samples() == 4
    cpu, _ = orc.render(64, 48, 4, 8, first_sample=0)
    assert match_fraction(a.film(), cpu) >= MIN_MATCH
    np.testing.assert_allclose(a.film(normalize=True), a.film() / 4, rtol=1e-6)
