"""CPU-only tests: the library loads and exports the declared C ABI, the
material JIT generates and NVRTC-compiles sm_100a code, codegen errors match
the oracle's, the oracle is stable against its committed golden vectors,
and the scene generators produce the configured sizes."""
import re
from pathlib import Path

import numpy as np
import pytest

import oracle_ctypes as O
from raymond_b200 import api, materials as M, scenes
from raymond_b200._abi import SceneDesc

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"


def declared_symbols():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        names += re.findall(r"^\s*(?:rmd_status|void|int32_t|const char \*)\s*(rmd_\w+)\s*\(", h.read_text(), re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(built):
    L = api.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(api.EXPORTS)
    assert b"sm_100a" in L.rmd_version()


def test_codegen_shape(built):
    src = api.generate_source(scenes.cornell(envmap_exponent=2), hoist=False)
    # the reference's code shape: Kernel<params> n{}; n.field = TYPE(value); n.compute(ctx, shading);
    assert "BsdfPrincipled<kBsdfPrincipled::DISTRIBUTION_GGX, kBsdfPrincipled::SUBSURFACE_METHOD_RANDOM_WALK>" in src
    assert "n1.baseColor = RGBA(make_float4(" in src
    assert "n1.normal = VECTOR(shading.normal);" in src
    assert "n0.surface = SHADER(n1.bsdf);" in src
    assert "void shadeSurface(" in src and "void shadeLight(" in src


def test_codegen_hoisting_shares_structure(built):
    sc = scenes.spheres_terrain(seed=2, num_spheres=5, terrain_cells=4, envmap_exponent=2)
    src = api.generate_source(sc, hoist=True)
    # 6 materials with the same graph structure -> one function
    assert src.count("__device__ __forceinline__ void s_") == 1
    assert "TexNoise<kTexNoise::DIMENSION_3D>" in src and "ColorRamp<2>" in src


def test_jit_compiles_for_sm100a(built):
    nbytes, log = api.jit_compile(scenes.spheres_terrain(seed=2, num_spheres=3, terrain_cells=4, envmap_exponent=2))
    assert nbytes > 10000


def _scene_with(graph):
    sc = scenes.cornell(envmap_exponent=2)
    sc["materials"][0] = ("broken", graph)
    return SceneDesc(sc)


@pytest.mark.parametrize("case,status", [("cycle", 4), ("multi", 5), ("unsupported", 6)])
def test_codegen_errors_match_oracle(built, case, status):
    g = M.principled()
    if case == "cycle":
        g["Mix"] = {"type": "MIX", "inputs": {"A_Color": {"type": "RGBA", "links": [["Mix2", "Result_Color"]]}},
                    "parameters": {}}
        g["Mix2"] = {"type": "MIX", "inputs": {"A_Color": {"type": "RGBA", "links": [["Mix", "Result_Color"]]}},
                     "parameters": {}}
        g["Principled BSDF"]["inputs"]["Base Color"] = {"type": "RGBA", "links": [["Mix", "Result_Color"]]}
    elif case == "multi":
        g["Principled BSDF"]["inputs"]["Base Color"] = {
            "type": "RGBA", "links": [["Principled BSDF", "BSDF"], ["Principled BSDF", "BSDF"]]}
    else:
        g["Principled BSDF"]["type"] = "BSDF_HAIR_PRINCIPLED"
    desc = _scene_with(g)
    with pytest.raises(api.RmdError) as e:
        api.generate_source(desc)
    assert e.value.status == status
    with pytest.raises(RuntimeError, match=f"\\({status}\\)"):
        O.OracleScene(desc)


def test_make_identifier_rules(built):
    # MaterialBuilder.swift:19-30,41-43 on the socket names the configs use
    src = api.generate_source(scenes.spheres_terrain(seed=2, num_spheres=1, terrain_cells=2, envmap_exponent=2),
                              hoist=False)
    for field in ["factor_Float", "a_Color", "b_Color", "subsurfaceIor", "emissionStrength", "ior", "fac"]:
        assert f".{field} = " in src, field
    assert "ColorRamp" in src and ".result_Color" in src


def test_scene_sizes():
    assert scenes.triangle_count(scenes.cornell()) == 36
    sc = scenes.spheres_terrain(num_spheres=64, subdivisions=5, terrain_cells=512)
    assert scenes.triangle_count(sc) == 64 * 5120 + 2 * 512 * 512
    assert len(sc["point_lights"]) == 16 and len(sc["sun_lights"]) == 1


def test_oracle_golden_prng():
    data = np.load(GOLDEN / "prng.npz")
    for key in data.files:
        mode, a, b = (int(x) for x in key.split("_")[1:])
        assert np.array_equal(O.prng(mode, a, b, len(data[key])).view(np.uint32), data[key].view(np.uint32)), key


def test_oracle_golden_cornell():
    """The oracle's Cornell box (64x64, 4 samples, PCG32 seed 1) is unchanged."""
    data = np.load(GOLDEN / "cornell_64.npz")
    orc = O.OracleScene(SceneDesc(scenes.cornell(seed=1, envmap_exponent=4)))
    film, st = orc.render(64, 64, 4, 8)
    np.testing.assert_allclose(film, data["film"], rtol=1e-5, atol=1e-7)
    assert st["segments"] == int(data["segments"])


def test_oracle_golden_noise():
    data = np.load(GOLDEN / "noise.npz")
    got = O.fractal_noise3(data["p"], 2.0, 0.5)
    assert np.array_equal(got.view(np.uint32), data["v"].view(np.uint32))


def test_oracle_energy_white_furnace():
    """Closed white diffuse room lit by its emissive walls (every surface emits 1,
    albedo 0.5, MIS): the radiance converges to 1 / (1 - 0.5) = 2 only in the
    limit of infinite depth; with depth 8 the geometric sum gives 2(1 - 0.5^8)."""
    sc = scenes.cornell(envmap_exponent=2)
    g = M.principled(base_color=(0.5, 0.5, 0.5, 1.0), roughness=1.0, emission=(1.0, 1.0, 1.0, 1.0),
                     emission_strength=1.0)
    g["Principled BSDF"]["inputs"]["Specular"]["value"] = 0.0
    sc["materials"] = [(n, g) for n, _ in sc["materials"]]
    # close the box: add a front wall facing the inside (the camera sits inside the room)
    sc["shapes"].append(scenes.quad_mesh(np.array([[0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.float32),
                                         [0, 0, -1], 0))
    sc["entities"].append({"shape": len(sc["shapes"]) - 1, "matrix": np.eye(4)})
    sc["camera"]["transform"] = scenes.look_at((0.5, 0.5, 0.9), (0.5, 0.5, 0.0))
    film, _ = O.OracleScene(SceneDesc(sc)).render(16, 16, 64, 8)
    mean = film.mean() / 64
    assert 1.5 < mean < 2.1, mean


@pytest.mark.parametrize("name", ["glossy_room", "glossy_rooms_grid"])
def test_oracle_bvh_culling_keeps_the_closest_hit(name):
    """The oracle's BVH culls boxes against the best hit so far with a widened
    bound; its closest hits equal those of the exhaustive search (every box
    the ray enters) bit for bit, on random rays and on rays leaving surfaces,
    in scenes with coplanar shared walls and boxes standing on floors.  (With
    an unwidened bound 6e-4 of the random and 1e-3 of the secondary rays in
    the glossy room returned a farther face.)"""
    d = getattr(scenes, name)(seed=1)
    orc = O.OracleScene(SceneDesc(d))
    v = np.concatenate([np.asarray(d["shapes"][e["shape"]]["vertices"], np.float64).reshape(-1, 3)
                        @ np.asarray(e["matrix"], np.float64)[:3, :3].T + np.asarray(e["matrix"], np.float64)[:3, 3]
                        for e in d["entities"]])
    rng = np.random.default_rng(11)
    n = 100000
    o = rng.uniform(v.min(0), v.max(0), (n, 3))
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 4:7], rays[:, 7] = o, dirs, 1e30
    h, _ = orc.trace(rays)
    hit = h[:, 0] > 0
    second = np.zeros((int(hit.sum()), 8), np.float32)
    second[:, 0:3] = o[hit] + dirs[hit] * h[hit, 0:1]
    d2 = rng.normal(size=(len(second), 3))
    second[:, 4:7] = d2 / np.linalg.norm(d2, axis=1, keepdims=True)
    second[:, 3], second[:, 7] = 1e-4, 1e30
    for r in (rays, second):
        a, ia = orc.trace(r)
        b, ib = orc.trace(r, exhaustive=True)
        assert (a[:, 0] > 0).mean() > 0.5
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        np.testing.assert_array_equal(ia, ib)


def test_oracle_scenes_are_independent():
    """A scene built after others were destroyed renders exactly as a fresh one
    (the oracle's per-thread node scratch must not outlive its program)."""
    import gc

    from test_parity_gpu import _all_lights_scene

    desc = SceneDesc(_all_lights_scene())
    ref, _ = O.OracleScene(desc).render(32, 32, 1, 4, sampling_mode=1)
    for seed in range(3):
        other = O.OracleScene(SceneDesc(scenes.cornell(seed=seed, envmap_exponent=4)))
        other.render(16, 16, 1, 4)
        del other
        gc.collect()
        again, _ = O.OracleScene(desc).render(32, 32, 1, 4, sampling_mode=1)
        assert np.array_equal(again, ref), seed


def test_bench_parity_time_interpolation():
    """bench.py's guided legs report the time a relMSE curve reaches the plain
    tracer's error: the first chunk at or below it, and the crossing
    interpolated in log relMSE between that chunk and the one before."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    curve = [(32, 100.0, 0.01), (64, 200.0, 0.005), (96, 300.0, 0.0033)]
    t = b.crossing_ms(curve, 0.004)
    assert 200.0 < t < 300.0
    assert abs(t - (200.0 + 100.0 * np.log(0.005 / 0.004) / np.log(0.005 / 0.0033))) < 1e-9
    assert b.crossing_ms(curve, 0.02) == 100.0  # reached by the first chunk
    assert b.crossing_ms(curve, 0.001) is None  # never reached
