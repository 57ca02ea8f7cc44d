"""Batched rendering: many scenes and views in one wavefront and one
CUDA-graph launch.  Each view must render exactly as it does alone (same
camera rays, same PCG stream of its own pixel index): per-sample radiance is
compared with the single-view renderer under the image parity criterion
(|batch - single| <= 1e-3 |single| + 1e-6 on >= 99.9 % of pixels; in
practice bit-identical)."""
import numpy as np
import pytest

from raymond_b200 import api, scenes
from raymond_b200._abi import SceneDesc
from raymond_b200.scenes import look_at

pytestmark = pytest.mark.gpu


def _match(a, b):
    ok = np.abs(a.astype(np.float64) - b) <= 1e-3 * np.abs(b) + 1e-6
    return float(ok.all(axis=-1).mean())


@pytest.fixture(scope="module")
def batch_setup(gpu_ctx):
    descs = [SceneDesc(scenes.cornell(seed=1, envmap_exponent=6)),
             SceneDesc(scenes.cornell_all_lights(seed=4, envmap_exponent=6))]
    side = {"transform": look_at((0.9, 0.6, 1.8), (0.4, 0.3, 0.3)), "near_clip": 1e-3, "far_clip": 100.0,
            "focal_length": 1.5, "shift": (0.0, 0.0)}
    views = [{"scene": 0, "width": 96, "height": 64},
             {"scene": 1, "width": 80, "height": 80},
             {"scene": 0, "width": 50, "height": 37, "camera": side}]
    return descs, views


def _single(gpu_ctx, desc, view, spp, first, **kw):
    scene = api.Scene(gpu_ctx, desc)
    r = api.Renderer(scene, view["width"], view["height"])
    if "camera" in view:
        r.set_camera(view["camera"])
    r.render(spp=spp, first_sample=first, **kw)
    return r.film()


@pytest.mark.parametrize("graph", [True, False])
def test_batch_views_match_single_renders(gpu_ctx, batch_setup, graph):
    descs, views = batch_setup
    b = api.Batch(gpu_ctx, descs, views, graph=graph)
    for first in (0, 5):
        b.reset()
        b.render(spp=1, max_depth=8, first_sample=first)
        st = b.stats()
        assert st["paths"] == sum(v["width"] * v["height"] for v in views)
        for i, v in enumerate(views):
            single = _single(gpu_ctx, descs[v["scene"]], v, 1, first, max_depth=8)
            assert _match(b.film(i), single) >= 0.999, (graph, first, i)


def test_batch_graph_equals_host_loop_and_accumulates(gpu_ctx, batch_setup):
    descs, views = batch_setup
    g = api.Batch(gpu_ctx, descs, views, graph=True)
    h = api.Batch(gpu_ctx, descs, views, graph=False)
    for b in (g, h):
        b.render(spp=3, max_depth=8)
        b.render(spp=5, max_depth=8)  # continues at sample 3
    for i, v in enumerate(views):
        # several samples per pixel: the film's float atomics add in a different order
        assert np.allclose(g.film(i), h.film(i), rtol=1e-5, atol=1e-6), i
        single = _single(gpu_ctx, descs[v["scene"]], v, 8, 0, max_depth=8)
        assert np.allclose(g.film(i), single, rtol=1e-4, atol=1e-5), i
    assert g.stats()["iterations"] >= 2 and g.stats()["errors"] == 0


def _textured_cornell(seed, textures):
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "ref"))
    import pin_materials

    sc = scenes.cornell(seed=seed, envmap_exponent=6)
    base = len(sc["materials"])
    sc["materials"] = sc["materials"] + [("textured", dict(pin_materials.materials())["image_textures"])]
    sc["textures"] = textures
    for sh in sc["shapes"][:-1]:
        sh["materials"] = np.full_like(sh["materials"], base)
    return sc


def test_batch_with_textures(gpu_ctx):
    """Textured scenes in one batch: every scene's image nodes read its own
    textures (a file another scene has but this one lacks reads the zero
    texture; one name may mean different images in two scenes), and each view
    renders as it does alone."""
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "ref"))
    import pin_materials

    tex = pin_materials.textures()
    lacking = {k: v for k, v in tex.items() if k != "textures/sky.exr"}
    other = dict(tex)
    other["textures/albedo.png"] = tex["textures/albedo.png"][::-1].copy()  # same name, another image
    descs = [SceneDesc(_textured_cornell(1, tex)), SceneDesc(_textured_cornell(2, lacking)),
             SceneDesc(_textured_cornell(3, other))]
    views = [{"scene": 0, "width": 64, "height": 48}, {"scene": 1, "width": 40, "height": 40},
             {"scene": 2, "width": 48, "height": 32}]
    b = api.Batch(gpu_ctx, descs, views)
    b.render(spp=1, max_depth=8, first_sample=3)
    for i, v in enumerate(views):
        single = _single(gpu_ctx, descs[v["scene"]], v, 1, 3, max_depth=8)
        assert _match(b.film(i), single) >= 0.999, i


def test_batch_rejects_bad_views(gpu_ctx, batch_setup):
    descs, views = batch_setup
    with pytest.raises(api.RmdError):
        api.Batch(gpu_ctx, descs, [{"scene": 2, "width": 8, "height": 8}])
    with pytest.raises(api.RmdError):
        api.Batch(gpu_ctx, descs, [{"scene": 0, "width": 0, "height": 8}])


def test_batch_guiding(gpu_ctx, batch_setup):
    """Guiding in a batch whose views show one scene: training runs (host
    loop), sampling-only renders run in the graph, and both converge to the
    plain tracer's images; a batch over two scenes refuses the guide."""
    descs, views = batch_setup
    with pytest.raises(api.RmdError):
        api.Batch(gpu_ctx, descs, views).set_guide()
    one = [v for v in views if v["scene"] == 0]
    b = api.Batch(gpu_ctx, descs[:1], one)
    b.set_guide(sampling=True, training=True, batch_size=1 << 14, steps_per_batch=4, seed=3)
    b.render(spp=1024, max_depth=8, seed=2, film_fp64=True)
    st = b.guide_stats()
    assert st["steps"] > 10 and np.isfinite(st["last_loss"])
    b.set_guide(sampling=True, training=False, batch_size=1 << 14)
    b.render(spp=1024, max_depth=8, seed=3, film_fp64=True)  # graph launch with inference inside
    for i, v in enumerate(one):
        plain = api.Renderer(api.Scene(gpu_ctx, descs[0]), v["width"], v["height"])
        if "camera" in v:
            plain.set_camera(v["camera"])
        plain.render(spp=2048, max_depth=8, seed=1, film_fp64=True)
        a = plain.film64() / 2048
        g = b.film64(i) / 2048
        assert abs(g.mean() / a.mean() - 1) < 0.02, (i, a.mean(), g.mean())
