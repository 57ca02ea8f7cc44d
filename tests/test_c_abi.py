"""The C ABI from C: tests/c_abi/abi_cornell.c compiled against include/raymond.h.

On the CPU: the program prints the size, alignment and field offsets of every
struct the header declares; they must equal the Python ctypes mirror's, and
the host-facing records must have the layout of the reference's bridge
structs (Camera.hpp 96 B, lights/*.hpp, PerInstanceData.hpp 192 B,
Uniforms.hpp 64 B, as Swift and Metal lay them out).

On the GPU: the program builds a Cornell box lit by a shape light and one
record of each light type from C arrays, renders it through the ABI and
writes its images.  The same scene built in Python (cabi_scene) is rendered
by the oracle with the same PCG32 stream (per-pixel parity criterion, as in
the other parity tests: |gpu - cpu| <= 1e-3 |cpu| + 1e-6 on >= 99.9 % of
pixels) and by the Python API, whose film must equal the C program's.  The
frames driven by the reference's Uniforms (TEA, random seeds 1 and 2) are
normalised with exposure 1.5 and the Hable curve and compared with the
oracle's TEA frames through its normalizeImage restatement.
"""
import ctypes as C
import os
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle_ctypes as O
from raymond_b200 import _abi, api
from raymond_b200._abi import RNG_TEA, SAMPLING_MIS, TONEMAP_HABLE, VISIBLE_ALL, SceneDesc

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "c_abi" / "abi_cornell.c"
W = H = 96
REL, ABS, MIN_MATCH = 1e-3, 1e-6, 0.999

CTYPES = {
    "rmd_node_param": _abi.NodeParam, "rmd_node_input": _abi.NodeInput, "rmd_node": _abi.Node,
    "rmd_material": _abi.Material, "rmd_shape": _abi.Shape, "rmd_entity": _abi.Entity,
    "rmd_light_info": _abi.LightInfo, "rmd_area_light": _abi.AreaLight, "rmd_point_light": _abi.PointLight,
    "rmd_sun_light": _abi.SunLight, "rmd_spot_light": _abi.SpotLight, "rmd_camera": _abi.Camera,
    "rmd_per_instance_data": _abi.PerInstanceData, "rmd_uniforms": _abi.Uniforms, "rmd_texture": _abi.Texture,
    "rmd_scene_desc": _abi.SceneDescC, "rmd_render_settings": _abi.RenderSettings, "rmd_stats": _abi.Stats,
    "rmd_bvh_stats": _abi.BvhStats, "rmd_tune_result": _abi.TuneResult, "rmd_guide_settings": _abi.GuideSettings,
    "rmd_guide_stats": _abi.GuideStats, "rmd_batch_view": _abi.BatchView,
}
# the reference's bridge layout (sizes; field offsets are asserted in the library and below)
BRIDGE = {"rmd_camera": (96, 16), "rmd_light_info": (4, 2), "rmd_area_light": (96, 16),
          "rmd_point_light": (64, 16), "rmd_sun_light": (64, 16), "rmd_spot_light": (96, 16),
          "rmd_per_instance_data": (192, 16), "rmd_uniforms": (64, 4)}
BRIDGE_OFFSETS = {
    ("rmd_camera", "shift"): 80, ("rmd_area_light", "transform"): 16, ("rmd_area_light", "color"): 64,
    ("rmd_area_light", "is_circular"): 80, ("rmd_point_light", "color"): 48, ("rmd_sun_light", "color"): 48,
    ("rmd_spot_light", "color"): 64, ("rmd_spot_light", "spot_blend"): 84,
    ("rmd_per_instance_data", "bounds_min"): 32, ("rmd_per_instance_data", "normal_transform"): 128,
    ("rmd_per_instance_data", "visibility"): 176, ("rmd_uniforms", "sensor_scale"): 16,
    ("rmd_uniforms", "output_channel"): 60,
}


@pytest.fixture(scope="module")
def program(tmp_path_factory, built):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path_factory.mktemp("cabi") / "abi_cornell"
    lib_dir = ROOT / "raymond_b200"
    subprocess.run([cc, "-std=c11", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(SRC),
                    "-o", str(exe), "-L", str(lib_dir), "-lrmd", f"-Wl,-rpath,{lib_dir}"], check=True)
    return exe


def test_c_layout_matches_ctypes_and_bridge(program):
    out = subprocess.run([str(program), "layout"], check=True, capture_output=True, text=True).stdout
    sizes, offsets = {}, {}
    for line in out.splitlines():
        f = line.split()
        if f[0] == "struct":
            sizes[f[1]] = (int(f[2]), int(f[3]))
        else:
            offsets[(f[1], f[2])] = int(f[3])
    assert set(sizes) == set(CTYPES)
    for name, T in CTYPES.items():
        assert sizes[name][0] == C.sizeof(T), name
    for (name, field), off in offsets.items():
        assert getattr(CTYPES[name], field).offset == off, (name, field)
    for name, (size, align) in BRIDGE.items():
        assert sizes[name] == (size, align), name
    for key, off in BRIDGE_OFFSETS.items():
        assert offsets[key] == off, key


# ------------------------------------------------------------ the scene in Python

WALLS = [([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1]], [0, 1, 0]),
         ([[0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1]], [0, -1, 0]),
         ([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], [0, 0, 1]),
         ([[0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1]], [1, 0, 0]),
         ([[1, 0, 0], [1, 1, 0], [1, 1, 1], [1, 0, 1]], [-1, 0, 0])]
LAMP = ([[0.375, 0.999, 0.375], [0.625, 0.999, 0.375], [0.625, 0.999, 0.625], [0.375, 0.999, 0.625]], [0, -1, 0])
COLORS = [(0.7, 0.7, 0.7), (0.6, 0.6, 0.6), (0.5, 0.6, 0.7), (0.7, 0.2, 0.2), (0.2, 0.7, 0.3), (0.3, 0.3, 0.6)]
LO, HI = (0.2, 0.0, 0.3), (0.5, 0.4, 0.6)


def _mesh(quads):
    """abi_cornell.c's add_quad: four vertices per quad, two triangles turned to the quad's normal."""
    V, N, T, I, M = [], [], [], [], []
    for k, (v, n, mat) in enumerate(quads):
        v = np.asarray(v, np.float32)
        g = np.cross(v[1] - v[0], v[2] - v[0])
        flip = float(np.dot(g, n)) < 0
        b = 4 * k
        I += [[b, b + 2, b + 1], [b, b + 3, b + 2]] if flip else [[b, b + 1, b + 2], [b, b + 2, b + 3]]
        V += v.tolist()
        N += [list(n)] * 4
        T += [[0, 0], [1, 0], [1, 1], [0, 1]]
        M += [mat, mat]
    return {"vertices": np.array(V, np.float32), "normals": np.array(N, np.float32),
            "texcoords": np.array(T, np.float32), "indices": np.array(I, np.uint32),
            "materials": np.array(M, np.uint16)}


def _inp(t, v=None, link=None):
    d = {"type": t}
    if v is not None:
        d["value"] = v
    if link is not None:
        d["links"] = [list(link)]
    return d


def cabi_scene():
    mats = []
    for name, c in zip(["floor", "ceiling", "back", "left", "right", "box"], COLORS):
        mats.append((name, {
            "Principled BSDF": {"type": "BSDF_PRINCIPLED", "parameters": {},
                                "inputs": {"Base Color": _inp("RGBA", [*c, 1.0]), "Roughness": _inp("VALUE", 0.5),
                                           "Metallic": _inp("VALUE", 0.0), "Specular": _inp("VALUE", 0.5),
                                           "Normal": _inp("VECTOR", [0.0, 0.0, 0.0])}},
            "Material Output": {"type": "OUTPUT_MATERIAL", "parameters": {},
                                "inputs": {"Surface": _inp("SHADER", link=("Principled BSDF", "BSDF"))}}}))
    mats.append(("lamp_quad", {
        "Emission": {"type": "EMISSION", "parameters": {},
                     "inputs": {"Color": _inp("RGBA", [1.0, 1.0, 1.0, 1.0]), "Strength": _inp("VALUE", 15.0)}},
        "Material Output": {"type": "OUTPUT_MATERIAL", "parameters": {},
                            "inputs": {"Surface": _inp("SHADER", link=("Emission", "Emission"))}}}))
    world = {"Background": {"type": "BACKGROUND", "parameters": {},
                            "inputs": {"Color": _inp("RGBA", [0.0, 0.0, 0.0, 1.0]), "Strength": _inp("VALUE", 1.0)}},
             "World Output": {"type": "OUTPUT_WORLD", "parameters": {},
                              "inputs": {"Surface": _inp("SHADER", link=("Background", "Background"))}}}
    lamp = {"Emission": {"type": "EMISSION", "parameters": {},
                         "inputs": {"Color": _inp("RGBA", [1.0, 0.9, 0.8, 1.0]), "Strength": _inp("VALUE", 1.0)}},
            "Light Output": {"type": "OUTPUT_LIGHT", "parameters": {},
                             "inputs": {"Surface": _inp("SHADER", link=("Emission", "Emission"))}}}
    lo, hi = LO, HI
    box = [([[lo[0], lo[1], lo[2]], [hi[0], lo[1], lo[2]], [hi[0], lo[1], hi[2]], [lo[0], lo[1], hi[2]]], [0, -1, 0]),
           ([[lo[0], hi[1], lo[2]], [hi[0], hi[1], lo[2]], [hi[0], hi[1], hi[2]], [lo[0], hi[1], hi[2]]], [0, 1, 0]),
           ([[lo[0], lo[1], lo[2]], [hi[0], lo[1], lo[2]], [hi[0], hi[1], lo[2]], [lo[0], hi[1], lo[2]]], [0, 0, -1]),
           ([[lo[0], lo[1], hi[2]], [hi[0], lo[1], hi[2]], [hi[0], hi[1], hi[2]], [lo[0], hi[1], hi[2]]], [0, 0, 1]),
           ([[lo[0], lo[1], lo[2]], [lo[0], hi[1], lo[2]], [lo[0], hi[1], hi[2]], [lo[0], lo[1], hi[2]]], [-1, 0, 0]),
           ([[hi[0], lo[1], lo[2]], [hi[0], hi[1], lo[2]], [hi[0], hi[1], hi[2]], [hi[0], lo[1], hi[2]]], [1, 0, 0])]
    shapes = [_mesh([(v, n, k) for k, (v, n) in enumerate(WALLS)]), _mesh([(v, n, 5) for v, n in box]),
              _mesh([(LAMP[0], LAMP[1], 6)])]
    cam = np.eye(4, dtype=np.float32)
    cam[:3, 3] = (0.5, 0.5, 2.3)
    tr = np.array([[0.2, 0, 0, 0.5], [0, 0, 0.2, 0.95], [0, -0.2, 0, 0.5]], np.float32)
    return {
        "materials": mats, "light_materials": [("world", world), ("lamp", lamp)], "world_shader": 0,
        "envmap_exponent": 4, "shapes": shapes,
        "entities": [{"shape": i, "matrix": np.eye(4), "visibility": VISIBLE_ALL} for i in range(3)],
        "area_lights": [{"shader": 1, "transform": tr, "color": (4.0, 4.0, 4.0), "is_circular": True}],
        "point_lights": [{"shader": 1, "location": (0.3, 0.7, 0.6), "radius": 0.05, "color": (2.0, 2.0, 2.0)}],
        "spot_lights": [{"shader": 1, "location": (0.5, 0.9, 0.8), "direction": (0.0, -1.0, 0.0), "radius": 0.03,
                         "color": (6.0, 6.0, 6.0), "spot_size": 1.0, "spot_blend": 0.0}],
        "sun_lights": [{"shader": 1, "direction": (0.0, 0.6, 0.8), "angle": 0.0, "color": (1.0, 1.0, 1.0)}],
        "camera": {"transform": cam, "near_clip": 0.1, "far_clip": 100.0, "focal_length": 2.5},
    }


def cabi_desc() -> SceneDesc:
    """The descriptor with the light records' derived fields set to the C program's literals."""
    d = SceneDesc(cabi_scene())
    d.c.spot_lights[0].spot_size = 0.8
    d.c.spot_lights[0].spot_blend = 0.05
    d.c.sun_lights[0].direction[:3] = [0.0, 0.6, 0.8]
    d.c.sun_lights[0].cos_angle = 0.999
    return d


def test_cabi_scene_generates(built):
    """The Python twin compiles through the codegen (on the CPU)."""
    assert len(api.generate_source(cabi_desc())) > 0


@pytest.mark.gpu
def test_c_program_renders_cornell(program, tmp_path, gpu_ctx):
    out = tmp_path / "images.bin"
    env = dict(os.environ)
    res = subprocess.run([str(program), "render", str(out)], check=True, capture_output=True, text=True, env=env)
    raw = np.fromfile(out, np.float32)
    film = raw[:W * H * 3].reshape(H, W, 3)
    normalized = raw[W * H * 3:].reshape(H, W, 4)

    desc = cabi_desc()
    orc = O.OracleScene(desc)
    cpu, _ = orc.render(W, H, 1, 8, sampling_mode=SAMPLING_MIS, seed=1, first_sample=0)
    ok = np.abs(film.astype(np.float64) - cpu) <= REL * np.abs(cpu) + ABS
    assert ok.all(axis=-1).mean() >= MIN_MATCH
    assert film.sum() > 0

    # the same scene through the Python API: the same film
    scene = api.Scene(gpu_ctx, desc)
    r = api.Renderer(scene, W, H)
    r.render(spp=1, max_depth=8, first_sample=0, seed=1)
    np.testing.assert_array_equal(r.film(), film)

    # Uniforms-driven frames: TEA seeds 1 and 2, exposure 1.5, Hable, accumulated
    tea, _ = orc.render(W, H, 2, 8, sampling_mode=SAMPLING_MIS, rng=RNG_TEA, first_sample=0)
    ref = O.normalize_image(tea, 1.5, True, 1, TONEMAP_HABLE)
    ok = np.abs(normalized.astype(np.float64) - ref) <= REL * np.abs(ref) + ABS
    assert ok.all(axis=-1).mean() >= MIN_MATCH
    assert np.all(normalized[..., 3] == 1.0)

    # the per-instance records the program read back
    insts = [dict(zip(m.group(1).split()[0::2], m.group(1).split()[1::2]))
             for m in re.finditer(r"instance \d+ (.*)", res.stdout)]
    assert [int(i["vertex_offset"]) for i in insts] == [0, 20, 44]
    assert [int(i["face_offset"]) for i in insts] == [0, 10, 22]
    assert [int(i["light_index"]) for i in insts] == [-1, -1, 0]
    assert [int(i["light_face_count"]) for i in insts] == [0, 0, 2]
    mine = scene.instance_data()
    assert [m.vertex_offset for m in mine] == [0, 20, 44] and mine[2].light_index == 0
