"""The device BVH builder (rmd_context_set_bvh_builder(RMD_BVH_GPU)).

A BVH is correct when traversal finds every hit: every triangle sits in
exactly one leaf slot, its vertices lie inside every slot box on the path
from the root to that leaf (decoded in FP32, as the traversal kernels decode
them), every node is reached exactly once, and the tree is at most 32 levels
deep (the traversal stack).  These tests check that structure for the device-built
tree directly, then check that rays and renders through it match the host-built
tree's (and the oracle's BVH), on regular, random, degenerate and tiny inputs.
"""
import numpy as np
import pytest

from raymond_b200 import api, scenes
from raymond_b200._abi import SceneDesc

pytestmark = pytest.mark.gpu


def decode_nodes(raw: np.ndarray) -> dict[str, np.ndarray]:
    """80-byte nodes -> fields (the layout of device/traverse.cuh)."""
    raw = np.ascontiguousarray(raw, np.uint8)
    return {
        "origin": raw[:, 0:12].copy().view(np.float32).reshape(-1, 3),
        "exponent": raw[:, 12:15].astype(np.int32),
        "imask": raw[:, 15].astype(np.int32),
        "child_base": raw[:, 16:20].copy().view(np.uint32).reshape(-1),
        "tri_base": raw[:, 20:24].copy().view(np.uint32).reshape(-1),
        "meta": raw[:, 24:32].astype(np.int32),
        "qlo": raw[:, 32:56].reshape(-1, 3, 8).astype(np.float32),
        "qhi": raw[:, 56:80].reshape(-1, 3, 8).astype(np.float32),
    }


def slot_boxes(n: dict, i: int) -> tuple[np.ndarray, np.ndarray]:
    """Decoded child boxes (8, 3) of node i in FP32: origin + q * 2^(e - 127)."""
    scale = np.ldexp(np.float32(1), n["exponent"][i] - 127).astype(np.float32)
    lo = n["origin"][i][:, None] + n["qlo"][i] * scale[:, None]
    hi = n["origin"][i][:, None] + n["qhi"][i] * scale[:, None]
    return lo.T.astype(np.float32), hi.T.astype(np.float32)


def check_tree(raw: np.ndarray, tris: np.ndarray) -> int:
    """Asserts the structure described in the module docstring; returns the depth."""
    n = decode_nodes(raw)
    count = len(raw)
    seen_nodes = np.zeros(count, np.int32)
    seen_tris = np.zeros(len(tris), np.int32)
    verts = tris.reshape(-1, 3, 4)[:, :, :3]
    inf = np.float32(np.inf)
    stack = [(0, np.full(3, -inf, np.float32), np.full(3, inf, np.float32), 1)]
    depth = 0
    while stack:
        i, plo, phi, d = stack.pop()  # plo / phi: the intersection of the slot boxes above
        assert 0 <= i < count, i
        seen_nodes[i] += 1
        depth = max(depth, d)
        lo, hi = slot_boxes(n, i)
        inner = 0
        used_tri = []
        for c in range(8):
            is_inner = (n["imask"][i] >> c) & 1
            meta = n["meta"][i][c]
            if not is_inner and meta == 0:
                continue
            clo, chi = np.maximum(plo, lo[c]), np.minimum(phi, hi[c])
            if is_inner:
                stack.append((int(n["child_base"][i]) + inner, clo, chi, d + 1))
                inner += 1
            else:
                k = bin(meta >> 5).count("1")
                assert (meta >> 5) == (1 << k) - 1, meta  # unary count
                first = int(n["tri_base"][i]) + (meta & 31)
                for t in range(first, first + k):
                    used_tri.append(t)
                    seen_tris[t] += 1
                    v = verts[t]
                    assert np.all(v >= clo) and np.all(v <= chi), (i, c, t)
        assert len(used_tri) == len(set(used_tri))
    assert np.all(seen_nodes == 1), "every node reached exactly once"
    assert np.all(seen_tris == 1), "every triangle in exactly one leaf"
    assert depth <= 32
    return depth


def soup_scene(v: np.ndarray) -> dict:
    """A scene of the triangles v (n, 3, 3) with the Cornell box's materials and camera."""
    base = scenes.cornell(seed=1, envmap_exponent=7)
    v = np.asarray(v, np.float32).reshape(-1, 3, 3)
    n = len(v)
    nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
    mesh = {"vertices": v.reshape(-1, 3), "normals": np.repeat(nrm, 3, axis=0).astype(np.float32),
            "texcoords": np.zeros((3 * n, 2), np.float32),
            "indices": np.arange(3 * n, dtype=np.uint32).reshape(-1, 3),
            "materials": np.zeros(n, np.uint16)}
    base["shapes"] = [mesh]
    base["entities"] = [{"shape": 0, "matrix": np.eye(4), "visibility": base["entities"][0]["visibility"]}]
    return base


def both(desc_dict):
    desc = SceneDesc(desc_dict)
    host = api.Scene(api.Context(0, bvh_builder="host"), desc)
    gpu = api.Scene(api.Context(0, bvh_builder="gpu"), desc)
    return host, gpu


def random_rays(rng, lo, hi, n):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = 1e30
    return rays


def same_hits(a_scene, b_scene, rays):
    """Closest and any hits through two trees (or a tree and the oracle's
    BVH).  Boxes are culled against the best distance widened by the rounding
    of box planes and triangle distances, so each returns the closest hit of an
    exhaustive search, and equal distances go to the lower (instance,
    primitive): the records agree bit for bit, ties, duplicates and coplanar
    faces included."""
    a, ia = a_scene.trace(rays)
    b, ib = b_scene.trace(rays)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    np.testing.assert_array_equal(ia, ib)
    oa, _ = a_scene.trace(rays, any_hit=True)
    ob, _ = b_scene.trace(rays, any_hit=True)
    np.testing.assert_array_equal(oa[:, 0], ob[:, 0])


def secondary_rays(rng, scene, rays):
    """Rays leaving the closest hits of `rays` in random directions: origins on
    surfaces, where near-coincident faces (a box on the floor) are met."""
    h, _ = scene.trace(rays)
    hit = h[:, 0] > 0
    p = rays[hit, 0:3].astype(np.float64) + rays[hit, 4:7] * h[hit, 0:1]
    d = rng.normal(size=(len(p), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.zeros((len(p), 8), np.float32)
    out[:, 0:3] = p
    out[:, 3] = 1e-4
    out[:, 4:7] = d
    out[:, 7] = 1e30
    return out


def tiny_soups():
    rng = np.random.default_rng(3)
    out = {k: rng.uniform(-1, 1, (k, 3, 3)) for k in (1, 2, 3, 4, 5, 9, 100, 5000)}
    out["identical"] = np.tile(rng.uniform(-1, 1, (1, 3, 3)), (2000, 1, 1))
    out["same_centroid"] = rng.uniform(-1, 1, (3000, 3, 3)) * np.linspace(0.01, 1, 3000)[:, None, None]
    g = np.stack(np.meshgrid(np.arange(64), np.arange(64), indexing="ij"), -1).reshape(-1, 2).astype(np.float32)
    grid = np.zeros((len(g), 3, 3), np.float32)  # a regular grid of equal triangles: every cost ties
    grid[:, 0, [0, 2]] = g
    grid[:, 1, [0, 2]] = g + [1, 0]
    grid[:, 2, [0, 2]] = g + [0, 1]
    out["grid"] = grid
    out["zero_area"] = np.repeat(rng.uniform(-1, 1, (500, 1, 3)), 3, axis=1)
    return out


@pytest.mark.parametrize("name", list(tiny_soups()))
def test_gpu_bvh_soups(gpu_ctx, name):
    v = tiny_soups()[name]
    host, gpu = both(soup_scene(v))
    assert gpu.info()["triangles"] == host.info()["triangles"] == len(v)
    raw, tris = gpu.bvh_arrays()
    check_tree(raw, tris)
    # the same triangles as the host tree (instance, primitive, vertices)
    hraw, htris = host.bvh_arrays()
    key = lambda t: np.lexsort((t[:, 7].view(np.uint32), t[:, 3].view(np.uint32)))
    assert np.array_equal(tris[key(tris)], htris[key(htris)])
    st = gpu.bvh_stats()
    assert st["builder"] == "gpu" and st["nodes"] == len(raw) and st["levels"] <= 32
    lo, hi = v.reshape(-1, 3).min(0) - 0.5, v.reshape(-1, 3).max(0) + 0.5
    same_hits(host, gpu, random_rays(np.random.default_rng(5), lo, hi, 20000))


@pytest.fixture(scope="module")
def big_scenes(gpu_ctx):
    out = {}
    for name, d in [("spheres_terrain_small", scenes.spheres_terrain(seed=2, num_spheres=16, subdivisions=4,
                                                                      terrain_cells=128, envmap_exponent=7)),
                    ("glossy_room", scenes.glossy_room(seed=1))]:
        out[name] = (d, *both(d))
    return out


@pytest.mark.parametrize("name", ["spheres_terrain_small", "glossy_room"])
def test_gpu_bvh_scene_structure_and_quality(big_scenes, name):
    d, host, gpu = big_scenes[name]
    raw, tris = gpu.bvh_arrays()
    check_tree(raw, tris)
    hs, gs = host.bvh_stats(), gpu.bvh_stats()
    print(name, "host", hs, "gpu", gs)
    # the device tree's surface-area cost stays near the host's binned SAH
    assert gs["sah_cost"] <= 1.3 * hs["sah_cost"], (gs, hs)


@pytest.mark.parametrize("name", ["spheres_terrain_small", "glossy_room"])
def test_gpu_bvh_rays_match_host(big_scenes, name):
    d, host, gpu = big_scenes[name]
    raw, tris = gpu.bvh_arrays()
    v = tris.reshape(-1, 3, 4)[:, :, :3].reshape(-1, 3)
    rng = np.random.default_rng(11)
    rays = random_rays(rng, v.min(0), v.max(0), 200000)
    same_hits(host, gpu, rays)
    same_hits(host, gpu, secondary_rays(rng, host, rays))


def test_trees_match_oracle_bvh_on_shared_walls(gpu_ctx):
    """The 4 x 4 rooms: neighbouring rooms share coplanar walls, boxes stand on
    the floors, and hits lie close to origins on large faces.  Both device
    trees and the oracle's binary BVH return identical closest and any hits
    on random rays and on rays leaving surfaces."""
    import oracle_ctypes as O

    d = scenes.glossy_rooms_grid(seed=1)
    desc = SceneDesc(d)
    host, gpu = both(d)
    orc = O.OracleScene(desc)
    raw, tris = gpu.bvh_arrays()
    v = tris.reshape(-1, 3, 4)[:, :, :3].reshape(-1, 3)
    rng = np.random.default_rng(11)
    rays = random_rays(rng, v.min(0), v.max(0), 200000)
    second = secondary_rays(rng, orc, rays)
    for tree in (host, gpu):
        same_hits(orc, tree, rays)
        same_hits(orc, tree, second)


def test_gpu_bvh_render_matches_host(gpu_ctx):
    host, gpu = both(scenes.cornell(seed=1, envmap_exponent=7))
    imgs = []
    for sc in (host, gpu):
        r = api.Renderer(sc, 128, 128)
        r.render(spp=16, max_depth=8, seed=3)
        imgs.append(r.film())
    assert np.allclose(imgs[0], imgs[1], rtol=1e-4, atol=1e-6)


def test_bvh_builder_argument(gpu_ctx):
    with pytest.raises(ValueError):
        api.Context(0, bvh_builder="metal")
    with pytest.raises(api.RmdError):
        api.check(api.lib().rmd_context_set_bvh_builder(gpu_ctx.h, 7))
