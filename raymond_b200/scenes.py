"""Seeded procedural scenes for the benchmark configurations.

The reference ships no scenes (its author's scenes are not in the
repository), so every input is generated here from a seed with numpy's
PCG64 generator.  Each generator returns the scene dictionary consumed by
`raymond_b200._abi.SceneDesc` (and by the C ABI through it).

  cornell()        36-triangle Cornell box, emissive ceiling quad (radiance 15)
  spheres_terrain() 64 icospheres + fBm terrain, sun + 16 point lights, noise graph
  glossy_room()    10x10x4 closed room with furniture boxes, lit through a window
"""
from __future__ import annotations

import math
from typing import Any

import numpy as np

from . import materials as M
from ._abi import VISIBLE_ALL


# ----------------------------------------------------------------- helpers

def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Camera-to-world matrix (row-major); the camera looks down its -Z, +Y up."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = r, u, -f, eye
    return m


def translate_scale_rotate_y(t=(0, 0, 0), s=(1, 1, 1), angle=0.0) -> np.ndarray:
    c, sn = math.cos(angle), math.sin(angle)
    rot = np.array([[c, 0, sn, 0], [0, 1, 0, 0], [-sn, 0, c, 0], [0, 0, 0, 1]])
    sc = np.diag([s[0], s[1], s[2], 1.0])
    tr = np.eye(4)
    tr[:3, 3] = t
    return tr @ rot @ sc


def _orient(v: np.ndarray, idx: np.ndarray, want: np.ndarray) -> np.ndarray:
    """Flip faces whose geometric normal cross(v1-v0, v2-v0) disagrees with `want`."""
    n = np.cross(v[idx[:, 1]] - v[idx[:, 0]], v[idx[:, 2]] - v[idx[:, 0]])
    flip = np.einsum("ij,ij->i", n, want) < 0
    idx = idx.copy()
    idx[flip, 1], idx[flip, 2] = idx[flip, 2], idx[flip, 1].copy()
    return idx


def quad_mesh(corners: np.ndarray, normal, material: int) -> dict[str, Any]:
    """Two triangles over 4 corners (in order around the quad), flat normal."""
    v = np.asarray(corners, np.float32)
    n = np.tile(np.asarray(normal, np.float32), (4, 1))
    t = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    idx = _orient(v, idx, n[:2]).astype(np.uint32)
    return {"vertices": v, "normals": n, "texcoords": t, "indices": idx,
            "materials": np.full(2, material, np.uint16)}


def box_mesh(lo, hi, material: int) -> dict[str, Any]:
    """Axis-aligned box, 6 faces x 2 triangles, outward normals."""
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    faces = []
    for axis in range(3):
        for side, val in ((-1, lo[axis]), (1, hi[axis])):
            a, b = [k for k in range(3) if k != axis]
            c = np.zeros((4, 3), np.float32)
            c[:, axis] = val
            for i, (ua, ub) in enumerate(((0, 0), (1, 0), (1, 1), (0, 1))):
                c[i, a] = lo[a] if ua == 0 else hi[a]
                c[i, b] = lo[b] if ub == 0 else hi[b]
            nrm = np.zeros(3, np.float32)
            nrm[axis] = side
            faces.append(quad_mesh(c, nrm, material))
    return merge_meshes(faces)


def merge_meshes(meshes: list[dict[str, Any]]) -> dict[str, Any]:
    out: dict[str, list] = {k: [] for k in ("vertices", "normals", "texcoords", "indices", "materials")}
    base = 0
    for m in meshes:
        out["vertices"].append(m["vertices"])
        out["normals"].append(m["normals"])
        out["texcoords"].append(m["texcoords"])
        out["indices"].append(m["indices"] + base)
        out["materials"].append(m["materials"])
        base += len(m["vertices"])
    return {"vertices": np.concatenate(out["vertices"]).astype(np.float32),
            "normals": np.concatenate(out["normals"]).astype(np.float32),
            "texcoords": np.concatenate(out["texcoords"]).astype(np.float32),
            "indices": np.concatenate(out["indices"]).astype(np.uint32),
            "materials": np.concatenate(out["materials"]).astype(np.uint16)}


def icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere with Blender's subdivision count (1 = icosahedron, 20 faces;
    every further level splits each face in four: subdivisions=5 -> 5120 faces)."""
    p = (1 + 5 ** 0.5) / 2
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.asarray(x, np.float64) / np.linalg.norm(x) for x in v]
    faces = list(f)
    for _ in range(max(0, subdivisions - 1)):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.asarray(verts, np.float32)
    F = np.asarray(faces, np.uint32)
    F = _orient(V.astype(np.float64), F, V[F].mean(axis=1).astype(np.float64))
    return V, F.astype(np.uint32)


def sphere_mesh(V: np.ndarray, F: np.ndarray, material: int) -> dict[str, Any]:
    u = (np.arctan2(V[:, 2], V[:, 0]) / (2 * np.pi) + 0.5).astype(np.float32)
    w = (np.arccos(np.clip(V[:, 1], -1, 1)) / np.pi).astype(np.float32)
    return {"vertices": V, "normals": V.copy(), "texcoords": np.stack([u, w], 1),
            "indices": F, "materials": np.full(len(F), material, np.uint16)}


def fbm_heightfield(n: int, octaves: int, seed: int) -> np.ndarray:
    """(n+1)x(n+1) fractal sum of bilinearly interpolated value noise in [-1, 1]."""
    rng = np.random.default_rng(seed)
    h = np.zeros((n + 1, n + 1), np.float64)
    amp, total = 1.0, 0.0
    x = np.linspace(0, 1, n + 1)
    for o in range(octaves):
        res = 4 * 2 ** o
        lattice = rng.uniform(-1, 1, (res + 2, res + 2))
        gx = x * res
        i0 = np.floor(gx).astype(int)
        fx = gx - i0
        fx = fx * fx * (3 - 2 * fx)
        a = lattice[np.ix_(i0, i0)]
        b = lattice[np.ix_(i0 + 1, i0)]
        c = lattice[np.ix_(i0, i0 + 1)]
        d = lattice[np.ix_(i0 + 1, i0 + 1)]
        fxr = fx[:, None]
        fzr = fx[None, :]
        h += amp * ((a * (1 - fxr) + b * fxr) * (1 - fzr) + (c * (1 - fxr) + d * fxr) * fzr)
        total += amp
        amp *= 0.5
    return h / total


def terrain_mesh(cells: int, size: float, amplitude: float, octaves: int, seed: int, material: int):
    h = fbm_heightfield(cells, octaves, seed) * amplitude
    xs = np.linspace(0, size, cells + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    V = np.stack([X, h, Z], -1).reshape(-1, 3).astype(np.float32)
    dx = np.gradient(h, xs, axis=0)
    dz = np.gradient(h, xs, axis=1)
    N = np.stack([-dx, np.ones_like(h), -dz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    T = np.stack([X / size, Z / size], -1).reshape(-1, 2).astype(np.float32)
    i, j = np.meshgrid(np.arange(cells), np.arange(cells), indexing="ij")
    a = (i * (cells + 1) + j).reshape(-1)
    b = a + (cells + 1)
    c = b + 1
    d = a + 1
    F = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)]).astype(np.int64)
    F = _orient(V.astype(np.float64), F, np.tile([0.0, 1.0, 0.0], (len(F), 1)))
    return {"vertices": V, "normals": N.reshape(-1, 3).astype(np.float32), "texcoords": T,
            "indices": F.astype(np.uint32), "materials": np.full(len(F), material, np.uint16)}


def _identity():
    return np.eye(4)


# ----------------------------------------------------------------- configurations

def cornell(seed: int = 1, envmap_exponent: int = 11) -> dict[str, Any]:
    """Unit room (floor, ceiling, back, left, right walls), two boxes and a
    0.25 x 0.25 emissive ceiling quad of radiance 15: 36 triangles.  Every
    surface is Principled with base colour U[0.2, 0.8]^3, roughness 0.5,
    metallic 0; the world is black."""
    rng = np.random.default_rng(seed)
    mats = []
    shapes = []
    entities = []

    def add_material(name, graph):
        mats.append((name, graph))
        return len(mats) - 1

    walls = {
        "floor": ([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]], [0, 1, 0]),
        "ceiling": ([[0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1]], [0, -1, 0]),
        "back": ([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], [0, 0, 1]),
        "left": ([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1]], [1, 0, 0]),
        "right": ([[1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], [-1, 0, 0]),
    }
    for name, (corners, normal) in walls.items():
        m = add_material(name, M.principled(base_color=tuple(rng.uniform(0.2, 0.8, 3)), roughness=0.5, metallic=0.0))
        shapes.append(quad_mesh(np.asarray(corners, np.float32), normal, m))
        entities.append({"shape": len(shapes) - 1, "matrix": _identity(), "visibility": VISIBLE_ALL})
    for name, (size, pos, ang) in {"short_box": ((0.3, 0.3, 0.3), (0.33, 0.0, 0.62), 0.3),
                                   "tall_box": ((0.3, 0.6, 0.3), (0.66, 0.0, 0.33), -0.3)}.items():
        m = add_material(name, M.principled(base_color=tuple(rng.uniform(0.2, 0.8, 3)), roughness=0.5, metallic=0.0))
        sx, sy, sz = size
        shapes.append(box_mesh((-sx / 2, 0, -sz / 2), (sx / 2, sy, sz / 2), m))
        entities.append({"shape": len(shapes) - 1, "matrix": translate_scale_rotate_y(pos, (1, 1, 1), ang),
                         "visibility": VISIBLE_ALL})
    m = add_material("light", M.emission((1, 1, 1, 1), 15.0))
    y = 0.999
    shapes.append(quad_mesh(np.asarray([[0.375, y, 0.375], [0.625, y, 0.375], [0.625, y, 0.625],
                                        [0.375, y, 0.625]], np.float32), [0, -1, 0], m))
    entities.append({"shape": len(shapes) - 1, "matrix": _identity(), "visibility": VISIBLE_ALL})
    return {
        "name": "cornell",
        "materials": mats,
        "light_materials": [("world", M.world((0, 0, 0, 1), 1.0))],
        "world_shader": 0,
        "envmap_exponent": envmap_exponent,
        "shapes": shapes,
        "entities": entities,
        "camera": {"transform": look_at((0.5, 0.5, 2.3), (0.5, 0.5, 0.0)), "near_clip": 0.1, "far_clip": 100.0,
                   "focal_length": 2.5},
    }


def spheres_terrain(seed: int = 1, num_spheres: int = 64, subdivisions: int = 5, terrain_cells: int = 512,
                    num_point_lights: int = 16, envmap_exponent: int = 11) -> dict[str, Any]:
    """64 icospheres (Blender subdivisions=5: 5120 faces each) with centres
    U[0, 20]^3 and radius U[0.3, 1.5] on a 512 x 512-cell fBm terrain (4 octaves,
    amplitude 2) spanning 20 x 20: 327,680 + 524,288 = 851,968 triangles.
    Per object a Principled BSDF with roughness U[0.05, 1], metallic
    Bernoulli(0.3), base colour U[0, 1]^3, whose base colour is
    Noise(scale 5, detail 2) -> ColorRamp -> Mix(A = base colour).  One sun and
    16 point lights; black world."""
    rng = np.random.default_rng(seed)
    V, F = icosphere(subdivisions)
    mats, shapes, entities = [], [], []

    def material(i):
        return M.principled_noise_ramp(base_color=tuple(rng.uniform(0, 1, 3)), roughness=float(rng.uniform(0.05, 1.0)),
                                       metallic=float(rng.uniform() < 0.3))

    for i in range(num_spheres):
        mats.append((f"sphere{i}", material(i)))
        shapes.append(sphere_mesh(V, F, len(mats) - 1))
        c = rng.uniform(0, 20, 3)
        r = float(rng.uniform(0.3, 1.5))
        entities.append({"shape": len(shapes) - 1, "matrix": translate_scale_rotate_y(c, (r, r, r), 0.0),
                         "visibility": VISIBLE_ALL})
    mats.append(("terrain", material(num_spheres)))
    shapes.append(terrain_mesh(terrain_cells, 20.0, 2.0, 4, seed + 1000, len(mats) - 1))
    entities.append({"shape": len(shapes) - 1, "matrix": _identity(), "visibility": VISIBLE_ALL})
    lmats = [("world", M.world((0, 0, 0, 1), 1.0)), ("lamp", M.light((1, 1, 1, 1), 1.0))]
    points = []
    for i in range(num_point_lights):
        col = rng.uniform(0.5, 1.0, 3)
        points.append({"shader": 1, "location": tuple(rng.uniform([0, 4, 0], [20, 14, 20])), "radius": 0.0,
                       "color": tuple(col * 400.0)})
    suns = [{"shader": 1, "direction": (-0.4, 1.0, 0.3), "angle": 0.05, "color": (3.0, 2.9, 2.7)}]
    return {
        "name": "spheres_terrain",
        "materials": mats,
        "light_materials": lmats,
        "world_shader": 0,
        "envmap_exponent": envmap_exponent,
        "shapes": shapes,
        "entities": entities,
        "point_lights": points,
        "sun_lights": suns,
        "camera": {"transform": look_at((10.0, 13.0, 27.0), (10.0, 2.0, 9.0)), "near_clip": 0.1, "far_clip": 100.0,
                   "focal_length": 1.6},
    }


def triangle_count(scene: dict[str, Any]) -> int:
    return int(sum(len(scene["shapes"][e["shape"]]["indices"]) for e in scene["entities"]))


def cornell_all_lights(seed: int = 4, envmap_exponent: int = 7) -> dict[str, Any]:
    """The Cornell box lit by every light type of the reference (two area lights,
    one square and one circular; a point light with and one without radius; a
    spot light; a sun; the ceiling quad as a shape light) under a noise-textured
    world (Background colour from a 3D noise texture, so the environment
    importance map is not uniform); the room's open front lets paths escape."""
    sc = cornell(seed=seed, envmap_exponent=envmap_exponent)
    world = M.world((1.0, 1.0, 1.0, 1.0), 2.0)
    world["Noise Texture"] = {
        "type": "TEX_NOISE",
        "inputs": {"Vector": {"type": "VECTOR", "value": [0, 0, 0]}, "W": {"type": "VALUE", "value": 0.0},
                   "Scale": {"type": "VALUE", "value": 3.0}, "Detail": {"type": "VALUE", "value": 1.0},
                   "Roughness": {"type": "VALUE", "value": 0.5}, "Distortion": {"type": "VALUE", "value": 0.0}},
        "parameters": {"noise_dimensions": "3D"}}
    world["Background"]["inputs"]["Color"] = {"type": "RGBA", "links": [["Noise Texture", "Color"]]}
    lamp = M.light((1.0, 0.9, 0.8, 1.0), 1.0)
    sc["light_materials"] = [("world", world), ("lamp", lamp)]
    tr = np.array([[0.2, 0, 0, 0.5], [0, 0, 0.2, 0.95], [0, -0.2, 0, 0.5]], np.float32)  # facing down
    tr2 = tr.copy()
    tr2[0, 3] += 0.2
    sc["area_lights"] = [{"shader": 1, "transform": tr, "color": (4.0, 4.0, 4.0), "is_circular": False},
                         {"shader": 1, "transform": tr2, "color": (3.0, 2.0, 1.0), "is_circular": True}]
    sc["point_lights"] = [{"shader": 1, "location": (0.3, 0.7, 0.6), "radius": 0.05, "color": (2.0, 2.0, 2.0)},
                          {"shader": 1, "location": (0.7, 0.5, 0.7), "radius": 0.0, "color": (1.0, 1.5, 2.0)}]
    sc["spot_lights"] = [{"shader": 1, "location": (0.5, 0.9, 0.8), "direction": (0.0, -1.0, -0.3), "radius": 0.03,
                          "color": (6.0, 6.0, 6.0), "spot_size": 1.0, "spot_blend": 0.3}]
    sc["sun_lights"] = [{"shader": 1, "direction": (0.2, 0.3, 1.0), "angle": 0.1, "color": (1.0, 1.0, 1.0)}]
    sc["name"] = "cornell_all_lights"
    return sc


def _boxes_mesh(lo: np.ndarray, hi: np.ndarray, materials: np.ndarray, tess: int = 1) -> dict[str, Any]:
    """Many axis-aligned boxes in one mesh (vectorised box_mesh), each face a
    tess x tess grid of quads: 12 tess^2 outward-facing triangles per box."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    nb = lo.shape[0]
    g = np.linspace(0.0, 1.0, tess + 1, dtype=np.float32)
    u0, v0 = np.meshgrid(g[:-1], g[:-1], indexing="ij")
    u1, v1 = u0 + 1.0 / tess, v0 + 1.0 / tess
    cu = np.stack([u0, u1, u1, u0], -1).reshape(-1, 4)  # (tess^2, 4) quad corners in face coordinates
    cv = np.stack([v0, v0, v1, v1], -1).reshape(-1, 4)
    verts, norms = [], []
    for axis in range(3):
        a, b = [k for k in range(3) if k != axis]
        for side in (-1, 1):
            c = np.zeros((nb, tess * tess, 4, 3), np.float32)
            c[..., axis] = (lo if side < 0 else hi)[:, None, None, axis]
            c[..., a] = lo[:, None, None, a] + (hi - lo)[:, None, None, a] * cu[None]
            c[..., b] = lo[:, None, None, b] + (hi - lo)[:, None, None, b] * cv[None]
            nrm = np.zeros(3, np.float32)
            nrm[axis] = side
            verts.append(c)
            norms.append(np.broadcast_to(nrm, c.shape))
    nq = nb * 6 * tess * tess
    V = np.stack(verts, 1).reshape(nq * 4, 3)
    N = np.stack(norms, 1).reshape(nq * 4, 3).astype(np.float32)
    quad = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    idx = (np.arange(nq, dtype=np.uint32)[:, None, None] * 4 + quad[None]).reshape(-1, 3)
    idx = _orient(V, idx, N[idx[:, 0]])
    T = np.tile(np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32), (nq, 1))
    mats = np.repeat(np.asarray(materials, np.uint16), 12 * tess * tess)
    return {"vertices": V, "normals": N, "texcoords": T, "indices": idx.astype(np.uint32), "materials": mats}


def glossy_room(seed: int = 1, num_boxes: int = 136, tess: int = 11, num_materials: int = 64,
                envmap_exponent: int = 8) -> dict[str, Any]:
    """A closed 10 x 10 x 4 room lit only through a 0.5 x 0.5 window (in the
    wall z = 10) by an environment of constant radiance 5, furnished with
    random boxes standing on the floor or floating as shelves, each face
    tessellated into tess x tess quads (136 boxes of 1,452 triangles: 197,490
    triangles with the room).  Every surface is Principled with roughness
    U[0.02, 0.3], base colour U[0.2, 0.9]^3, metallic 0; boxes draw one of
    `num_materials` such materials.  The camera stands inside looking across
    the room towards the window."""
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(num_materials + 6):
        mats.append((f"glossy{i}", M.principled(base_color=tuple(rng.uniform(0.2, 0.9, 3)),
                                                 roughness=float(rng.uniform(0.02, 0.3)), metallic=0.0)))
    W, D, Hh = 10.0, 10.0, 4.0
    wx0, wx1, wy0, wy1 = 4.75, 5.25, 2.25, 2.75  # the window in the wall z = D
    walls = [
        quad_mesh([[0, 0, 0], [W, 0, 0], [W, 0, D], [0, 0, D]], [0, 1, 0], num_materials + 0),        # floor
        quad_mesh([[0, Hh, 0], [W, Hh, 0], [W, Hh, D], [0, Hh, D]], [0, -1, 0], num_materials + 1),   # ceiling
        quad_mesh([[0, 0, 0], [W, 0, 0], [W, Hh, 0], [0, Hh, 0]], [0, 0, 1], num_materials + 2),      # z = 0
        quad_mesh([[0, 0, 0], [0, Hh, 0], [0, Hh, D], [0, 0, D]], [1, 0, 0], num_materials + 3),      # x = 0
        quad_mesh([[W, 0, 0], [W, Hh, 0], [W, Hh, D], [W, 0, D]], [-1, 0, 0], num_materials + 4),     # x = W
    ]
    # wall z = D with the window hole: four quads around it
    for (x0, x1, y0, y1) in [(0, W, 0, wy0), (0, W, wy1, Hh), (0, wx0, wy0, wy1), (wx1, W, wy0, wy1)]:
        walls.append(quad_mesh([[x0, y0, D], [x1, y0, D], [x1, y1, D], [x0, y1, D]], [0, 0, -1], num_materials + 5))
    room = merge_meshes(walls)
    # furniture: footprint U[0.3, 1.2]^2, height U[0.2, 1.5]; 70 % stand on the
    # floor, 30 % float as shelves; the camera's surroundings are kept clear
    size = np.stack([rng.uniform(0.3, 1.2, num_boxes), rng.uniform(0.2, 1.5, num_boxes),
                     rng.uniform(0.3, 1.2, num_boxes)], 1).astype(np.float32)
    pos = np.stack([rng.uniform(0.1, W - 1.3, num_boxes), np.zeros(num_boxes),
                    rng.uniform(0.1, D - 1.3, num_boxes)], 1).astype(np.float32)
    floating = rng.uniform(0, 1, num_boxes) < 0.3
    pos[floating, 1] = rng.uniform(0.5, Hh - 1.6, floating.sum())
    near_cam = (np.abs(pos[:, 0] + 0.5 * size[:, 0] - 2.0) < 1.5) & (np.abs(pos[:, 2] + 0.5 * size[:, 2] - 1.5) < 1.5)
    pos[near_cam, 0] += 3.0
    hi = np.minimum(pos + size, [W - 0.05, Hh - 0.05, D - 0.05]).astype(np.float32)
    boxes = _boxes_mesh(pos, hi, rng.integers(0, num_materials, num_boxes), tess)
    ident = _identity()
    return {
        "name": "glossy_room",
        "materials": mats,
        "light_materials": [("world", M.world((1.0, 1.0, 1.0, 1.0), 5.0))],
        "shapes": [room, boxes],
        "entities": [{"shape": 0, "matrix": ident, "visibility": VISIBLE_ALL},
                     {"shape": 1, "matrix": ident, "visibility": VISIBLE_ALL}],
        "camera": {"transform": look_at((2.0, 1.6, 1.5), (6.0, 1.4, 9.0)), "near_clip": 1e-3,
                   "far_clip": 100.0, "focal_length": 1.2},
        "world_shader": 0,
        "envmap_exponent": envmap_exponent,
    }


def glossy_rooms_grid(seed: int = 1, grid: int = 4, boxes_per_room: int = 170, tess: int = 11,
                      num_materials: int = 64, emitters: int = 64, envmap_exponent: int = 8) -> dict[str, Any]:
    """grid x grid glossy rooms (each 10 x 10 x 4, a 0.5 x 0.5 window in its
    z-far wall onto an environment of radiance 5) side by side, furnished with
    seeded tessellated boxes (170 boxes of 1,452 triangles per room: about 4 M
    triangles for 4 x 4), surfaces Principled with roughness U[0.01, 0.5] and
    metallic Bernoulli(0.5), and `emitters` small emissive ceiling quads
    (0.05 x 0.05, radiance 500) spread over the rooms.  The scene's camera
    looks into the first room; `grid_views` gives cameras for the others."""
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(num_materials + 6):
        mats.append((f"mat{i}", M.principled(base_color=tuple(rng.uniform(0.2, 0.9, 3)),
                                             roughness=float(rng.uniform(0.01, 0.5)),
                                             metallic=float(rng.uniform() < 0.5))))
    emit = len(mats)
    mats.append(("emitter", M.emission((1.0, 1.0, 1.0, 1.0), 500.0)))
    W, D, Hh = 10.0, 10.0, 4.0
    shapes = []
    for gx in range(grid):
        for gz in range(grid):
            ox, oz = gx * W, gz * D
            walls = [
                quad_mesh([[ox, 0, oz], [ox + W, 0, oz], [ox + W, 0, oz + D], [ox, 0, oz + D]], [0, 1, 0], num_materials),
                quad_mesh([[ox, Hh, oz], [ox + W, Hh, oz], [ox + W, Hh, oz + D], [ox, Hh, oz + D]], [0, -1, 0],
                          num_materials + 1),
                quad_mesh([[ox, 0, oz], [ox + W, 0, oz], [ox + W, Hh, oz], [ox, Hh, oz]], [0, 0, 1], num_materials + 2),
                quad_mesh([[ox, 0, oz], [ox, Hh, oz], [ox, Hh, oz + D], [ox, 0, oz + D]], [1, 0, 0], num_materials + 3),
                quad_mesh([[ox + W, 0, oz], [ox + W, Hh, oz], [ox + W, Hh, oz + D], [ox + W, 0, oz + D]], [-1, 0, 0],
                          num_materials + 4),
            ]
            wx0, wx1, wy0, wy1, zD = ox + 4.75, ox + 5.25, 2.25, 2.75, oz + D
            for (x0, x1, y0, y1) in [(ox, ox + W, 0, wy0), (ox, ox + W, wy1, Hh), (ox, wx0, wy0, wy1),
                                     (wx1, ox + W, wy0, wy1)]:
                walls.append(quad_mesh([[x0, y0, zD], [x1, y0, zD], [x1, y1, zD], [x0, y1, zD]], [0, 0, -1],
                                       num_materials + 5))
            n = boxes_per_room
            size = np.stack([rng.uniform(0.3, 1.2, n), rng.uniform(0.2, 1.5, n), rng.uniform(0.3, 1.2, n)],
                            1).astype(np.float32)
            pos = np.stack([rng.uniform(0.1, W - 1.3, n), np.zeros(n), rng.uniform(0.1, D - 1.3, n)], 1).astype(np.float32)
            floating = rng.uniform(0, 1, n) < 0.3
            pos[floating, 1] = rng.uniform(0.5, Hh - 1.6, floating.sum())
            near_cam = (np.abs(pos[:, 0] + 0.5 * size[:, 0] - 2.0) < 1.5) & (np.abs(pos[:, 2] + 0.5 * size[:, 2] - 1.5) < 1.5)
            pos[near_cam, 0] += 3.0
            hi = np.minimum(pos + size, [W - 0.05, Hh - 0.05, D - 0.05]).astype(np.float32)
            pos += np.array([ox, 0, oz], np.float32)
            hi += np.array([ox, 0, oz], np.float32)
            shapes.append(merge_meshes(walls + [_boxes_mesh(pos, hi, rng.integers(0, num_materials, n), tess)]))
    # small emitters on the ceilings, facing down
    quads = []
    for e in range(emitters):
        cx, cz = rng.uniform(0.5, grid * W - 0.5), rng.uniform(0.5, grid * D - 0.5)
        y, h = Hh - 0.01, 0.025
        quads.append(quad_mesh([[cx - h, y, cz - h], [cx + h, y, cz - h], [cx + h, y, cz + h], [cx - h, y, cz + h]],
                               [0, -1, 0], emit))
    shapes.append(merge_meshes(quads))
    ident = _identity()
    return {
        "name": "glossy_rooms_grid",
        "materials": mats,
        "light_materials": [("world", M.world((1.0, 1.0, 1.0, 1.0), 5.0))],
        "shapes": shapes,
        "entities": [{"shape": i, "matrix": ident, "visibility": VISIBLE_ALL} for i in range(len(shapes))],
        "camera": grid_views(1, grid)[0],
        "world_shader": 0,
        "envmap_exponent": envmap_exponent,
    }


def grid_views(n: int, grid: int = 4) -> list[dict[str, Any]]:
    """n cameras of glossy_rooms_grid, each inside a different room looking
    across it towards its window."""
    out = []
    for k in range(n):
        gx, gz = k % grid, (k // grid) % grid
        ox, oz = gx * 10.0, gz * 10.0
        out.append({"transform": look_at((ox + 2.0, 1.6, oz + 1.5), (ox + 6.0, 1.4, oz + 9.0)), "near_clip": 1e-3,
                    "far_clip": 100.0, "focal_length": 1.2})
    return out
