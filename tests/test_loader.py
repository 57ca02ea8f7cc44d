"""Scene files in the reference's format (exporter JSON + ASCII PLY): the
reference's number parsing, round trips of the procedural scenes, and a
loaded scene rendered on the GPU against the oracle on the same file."""
import numpy as np
import pytest

from raymond_b200 import loader, scenes
from raymond_b200._abi import SceneDesc


def test_reference_float_parsing():
    toks = np.array(["0.100000", "-1.250000", "3", "-0.000000", "123456.789012"])
    got = loader.parse_reference_floats(toks)
    # integer of the digits times powf(10, -decimals), in float arithmetic
    want = np.array([np.float32(100000) * np.float32(1e-6), -(np.float32(1250000) * np.float32(1e-6)), np.float32(3),
                     np.float32(0), np.float32(123456789012) * np.float32(1e-6)], np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    with pytest.raises(loader.SceneFormatError):
        loader.parse_reference_floats(np.array(["1e-3"]))


@pytest.mark.parametrize("make", [lambda: scenes.cornell(seed=1), lambda: scenes.cornell_all_lights(seed=4)])
def test_round_trip(tmp_path, make):
    sc = make()
    loader.save_scene(sc, tmp_path / "scene.json", resolution=(64, 48))
    back, size = loader.load_scene(tmp_path / "scene.json")
    assert size == (64, 48)
    assert [n for n, _ in back["materials"]] == [n for n, _ in sc["materials"]]
    assert [n for n, _ in back["light_materials"]] == [n for n, _ in sc["light_materials"]]
    assert len(back["shapes"]) == len(sc["shapes"]) and len(back["entities"]) == len(sc["entities"])
    for a, b in zip(sc["shapes"], back["shapes"]):
        assert np.allclose(a["vertices"], b["vertices"], atol=1e-6)
        assert np.allclose(a["normals"], b["normals"], atol=1e-6)
        assert np.array_equal(np.asarray(a["indices"]), b["indices"])
        assert np.array_equal(np.asarray(a["materials"]), b["materials"])
    for key in ("area_lights", "point_lights", "sun_lights", "spot_lights"):
        assert len(back[key]) == len(sc.get(key, []))
        for a, b in zip(sc.get(key, []), back[key]):
            assert np.allclose(a["color"], b["color"], rtol=1e-6)
    assert np.allclose(np.asarray(back["camera"]["transform"]), np.asarray(sc["camera"]["transform"]), atol=1e-6)
    assert back["camera"]["focal_length"] == pytest.approx(sc["camera"]["focal_length"], rel=1e-6)
    SceneDesc(back)  # builds the C descriptor


def test_malformed_files(tmp_path):
    sc = scenes.cornell(seed=1)
    loader.save_scene(sc, tmp_path / "scene.json")
    ply = tmp_path / "meshes" / "shape0.ply"
    text = ply.read_text().replace("\n3 ", "\n4 ", 1)
    ply.write_text(text)
    with pytest.raises(loader.SceneFormatError):
        loader.load_scene(tmp_path / "scene.json")


@pytest.mark.gpu
def test_loaded_scene_matches_oracle(tmp_path, gpu_ctx):
    import oracle_ctypes as O
    from raymond_b200 import api
    loader.save_scene(scenes.cornell_all_lights(seed=4, envmap_exponent=6), tmp_path / "scene.json")
    sc, _ = loader.load_scene(tmp_path / "scene.json")
    sc["envmap_exponent"] = 6
    desc = SceneDesc(sc)
    r = api.Renderer(api.Scene(gpu_ctx, desc), 64, 64)
    orc = O.OracleScene(desc)
    for first in (0, 3):
        r.reset()
        r.render(spp=1, max_depth=8, first_sample=first)
        cpu, _ = orc.render(64, 64, 1, 8, first_sample=first)
        ok = np.abs(r.film().astype(np.float64) - cpu) <= 1e-3 * np.abs(cpu) + 1e-6
        assert ok.all(axis=-1).mean() >= 0.999
