"""Pinning the oracle against the reference's own device code.

The reference's Metal device library (PrngState, noise, the node structs, the
BSDF lobes and UberShader) is compiled for the host by oracle/ref/Makefile
against a Metal stand-in, and run on the same inputs as the oracle's
restatement.  tests/golden/ref_pin.npz holds its outputs (made by
tests/golden/make_ref_golden.py), so the comparison also runs where the
reference is not mounted; with the host build present the live test checks
fresh inputs too.

Bars: the TEA stream and fractal noise bit for bit; material evaluate/sample
results within the image parity tolerance (1e-3 relative, 1e-6 absolute) on
every record, and within 1e-5 relative on at least 99.5 % of them (the rest
differ by float rounding inside the sampling routines).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle_ctypes as O
from raymond_b200._abi import RNG_TEA, SceneDesc

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "ref"))
import pin_materials  # noqa: E402
import ref_ctypes as R  # noqa: E402

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_pin.npz"


@pytest.fixture(scope="module")
def oracle_pin_scene():
    return O.OracleScene(SceneDesc(pin_materials.scene()))


def _close_rows(a, b, rtol):
    ok = np.isclose(a, b, rtol=rtol, atol=1e-6) | (np.isnan(a) & np.isnan(b))
    return ok.all(axis=1)


def _check_materials(orc, records, ref_out, names):
    for m, name in enumerate(names):
        got = orc.material_eval(m, records)
        assert _close_rows(got, ref_out[m], 1e-3).all(), name
        assert _close_rows(got, ref_out[m], 1e-5).mean() >= 0.995, name
        # lobe flags and alpha exactly
        np.testing.assert_array_equal(got[:, 14], ref_out[m][:, 14], err_msg=name)
        np.testing.assert_array_equal(got[:, 15], ref_out[m][:, 15], err_msg=name)


def test_oracle_matches_reference_golden(oracle_pin_scene):
    g = np.load(GOLDEN)
    for (a, b), ref in zip(g["prng_cases"], g["prng"]):
        got = O.prng(RNG_TEA, int(a), int(b), ref.size)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (a, b)
    for (d, r), ref in zip(g["noise_cases"], g["noise"]):
        got = O.fractal_noise3(g["noise_points"], float(d), float(r))
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (d, r)
    names = [str(n) for n in g["material_names"]]
    assert names == [n for n, _ in pin_materials.materials()]
    _check_materials(oracle_pin_scene, g["records"], g["materials"], names)


@pytest.mark.skipif(not R.available(), reason="host build of the reference (oracle/_ref/libref.so) not present")
def test_oracle_matches_reference_live(oracle_pin_scene):
    for a, b in [(3, 5), (2**31 + 11, 17), (65536, 1)]:
        assert np.array_equal(R.prng_tea(a, b, 300).view(np.uint32), O.prng(RNG_TEA, a, b, 300).view(np.uint32))
    pts = np.random.default_rng(9).uniform(-1e3, 1e3, (4096, 3)).astype(np.float32)
    for d, r in [(1.0, 0.3), (6.25, 0.55)]:
        assert np.array_equal(R.fractal_noise3(pts, d, r).view(np.uint32), O.fractal_noise3(pts, d, r).view(np.uint32))
    pin_materials.install_ref_textures(R)
    rec = R.shading_records(2048, seed=77)
    names = [n for n, _ in pin_materials.materials()]
    ref_out = np.stack([R.material_eval(m, rec) for m in range(len(names))])
    _check_materials(oracle_pin_scene, rec, ref_out, names)


# ---------------------------------------------------------------- whole images
# One-sample images rendered by the reference's own kernels (host build, TEA
# generator as generateRays seeds it) against the oracle's TEA mode: the same
# per-sample parity bar as the GPU tests.
RENDER_GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_render.npz"
REL, ABS, MIN_MATCH = 1e-3, 1e-6, 0.999


def _match(ref_film, cpu):
    ref = ref_film[..., :3].astype(np.float64)
    ok = np.abs(ref - cpu) <= REL * np.abs(cpu) + ABS
    return float(ok.all(axis=-1).mean())


@pytest.fixture(scope="module")
def ref_scene_descs():
    return {k: SceneDesc(v) for k, v in pin_materials.ref_scenes().items() if k != "pin"}


def test_oracle_images_match_reference_golden(ref_scene_descs):
    g = np.load(RENDER_GOLDEN)
    cases = {}
    for key in g.files:
        name, rest = key.split("/", 1)
        if rest != "size":
            cases.setdefault(name, []).append(key)
    assert set(cases) == {"cornell", "cornell_all_lights", "spheres_small"}
    for name, keys in cases.items():
        w, h, depth = (int(x) for x in g[f"{name}/size"])
        orc = O.OracleScene(ref_scene_descs[name])
        for key in keys:
            _, mode, frame = key.split("/")
            cpu, _ = orc.render(w, h, 1, depth, sampling_mode=int(mode), rng=RNG_TEA, first_sample=int(frame))
            assert _match(g[key], cpu) >= MIN_MATCH, key


@pytest.mark.skipif(not R.available(), reason="host build of the reference (oracle/_ref/libref.so) not present")
@pytest.mark.parametrize("name", ["cornell", "cornell_all_lights", "spheres_small"])
def test_oracle_images_match_reference_live(ref_scene_descs, name):
    desc = ref_scene_descs[name]
    orc = O.OracleScene(desc)
    ref = R.RefScene(desc, name, orc.surface_emissive())
    for mode in (0, 1, 2):
        for frame in (2, 9):
            rf = ref.render(40, 30, 1, 10, sampling_mode=mode, first_frame=frame)
            cpu, _ = orc.render(40, 30, 1, 10, sampling_mode=mode, rng=RNG_TEA, first_sample=frame)
            assert _match(rf, cpu) >= MIN_MATCH, (mode, frame)


# ------------------------------------------------------------------ tonemapping
# normalizeImage (normalizeImage.metal:11-59): the oracle's restatement against
# the reference's own kernel, bit for bit.
TONEMAP_GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_tonemap.npz"


def test_oracle_tonemap_matches_reference_golden():
    g = np.load(TONEMAP_GOLDEN)
    for (e, a, f, t), ref in zip(g["cases"], g["images"]):
        got = O.normalize_image(g["film"], float(e), bool(a), int(f), int(t))
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (e, a, f, t)


@pytest.mark.skipif(not R.available(), reason="host build of the reference (oracle/_ref/libref.so) not present")
def test_oracle_tonemap_matches_reference_live():
    film = np.random.default_rng(4).gamma(0.5, 4.0, (23, 31, 4)).astype(np.float32)
    for t in (0, 1, 2):
        for e, a, f in ((2.5, 1, 3), (1.0, 0, 9)):
            ref = R.normalize_image(film, e, bool(a), f, t)
            got = O.normalize_image(film, e, bool(a), f, t)
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (t, e, a, f)


# ------------------------------------------------------------------ Nishita sky
# The sky texture and sun disc of the TEX_SKY node (host/sky/sky_nishita.cpp):
# the oracle's restatement against the reference's own model, bit for bit.
SKY_GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_sky.npz"


def test_oracle_sky_matches_reference_golden():
    g = np.load(SKY_GOLDEN)
    n = g["textures"].shape[1]
    for (e, alt, air, dust, oz, rot, size, inten), tex, sun in zip(g["cases"], g["textures"], g["sun"]):
        got = O.sky_texture(n, n, e, alt, air, dust, oz)[..., :3]
        assert np.array_equal(got.view(np.uint32), tex.view(np.uint32)), (e, alt)
        data = O.sky_data(e, rot, True, size, inten, alt, air, dust)
        assert np.array_equal(data[:6].view(np.uint32), sun.view(np.uint32)), (e, alt)
        assert list(data[6:]) == [np.float32(e), np.float32(rot), np.float32(size), np.float32(inten)]


@pytest.mark.skipif(not R.sky_available(), reason="host build of the reference's sky model not present")
def test_oracle_sky_matches_reference_live():
    for args in [(0.7, 300.0, 1.1, 0.9, 1.3), (0.01, 0.0, 1.0, 1.0, 1.0)]:
        ref = R.sky_texture(96, 80, *args)
        got = O.sky_texture(96, 80, *args)[..., :3]
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), args
