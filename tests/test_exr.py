"""OpenEXR output (rmd_film_save_exr), the headless form of the reference's
MTLTexture.saveEXR (utils/Metal.swift:75-126).

The writer is checked three ways on the CPU: its files read back exactly with
the package's reader; they load with the reference's own EXR library
(tinyexr, raymond/io/tinyexr.cpp, built by oracle/ref/Makefile into
oracle/_ref/libtinyexr.so) to the same floats; and files that tinyexr's
SaveEXR writes from the same pixels - as the reference does - carry the same
channels, compression and values.  A GPU test saves a rendered film.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from raymond_b200 import api, exr, scenes
from raymond_b200._abi import SceneDesc

TINYEXR = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libtinyexr.so"


def image(h, w, seed=0):
    rng = np.random.default_rng(seed)
    img = rng.exponential(1.0, (h, w, 3)).astype(np.float32)
    img[0, 0] = [0.0, -1.5, 1e30]  # zero, negative, huge
    if h * w > 4:
        img[-1, -1] = [np.float32(1e-42), 3.0, 7.25]  # a subnormal
    return img


SIZES = [(1, 1), (3, 7), (15, 15), (16, 16), (17, 33), (64, 48)]


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("compression", ["auto", "none", "zip"])
def test_exr_round_trip(built, tmp_path, h, w, compression):
    img = image(h, w)
    p = tmp_path / "f.exr"
    api.test_exr_write(p, img, normalized_by=0.25, compression=compression)
    rgba = exr.read_rgba(p)
    expect = img * np.float32(0.25)
    assert np.array_equal(rgba[..., :3].view(np.uint32), expect.view(np.uint32))
    assert np.all(rgba[..., 3] == 1.0)
    _, header = exr.read_exr(p)
    assert [c for c, _ in header["channels"]] == ["A", "B", "G", "R"]
    assert all(t == 2 for _, t in header["channels"])  # FLOAT
    zipped = compression == "zip" or (compression == "auto" and not (w < 16 and h < 16))
    assert header["compression"] == (3 if zipped else 0)
    assert header["dataWindow"] == (0, 0, w - 1, h - 1)


def test_exr_errors(built, tmp_path):
    with pytest.raises(ValueError):
        api.test_exr_write(tmp_path / "x.exr", image(2, 2), compression="rle")
    with pytest.raises(api.RmdError):
        api.test_exr_write(tmp_path / "missing_dir" / "x.exr", image(2, 2))
    with pytest.raises(api.RmdError):
        api.check(api.lib().rmd_test_exr_write(str(tmp_path / "x.exr").encode(),
                                               image(2, 2).ctypes.data_as(C.POINTER(C.c_float)), 2, 2, 1.0, 9))


def tinyexr():
    if not TINYEXR.exists():
        pytest.skip("oracle/_ref/libtinyexr.so not built (needs the reference's sources)")
    L = C.CDLL(str(TINYEXR))
    L.LoadEXR.argtypes = [C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p,
                          C.POINTER(C.c_char_p)]
    L.SaveEXR.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p,
                          C.POINTER(C.c_char_p)]
    return L


@pytest.mark.parametrize("h,w", SIZES)
def test_exr_loads_in_reference_library(built, tmp_path, h, w):
    L = tinyexr()
    img = image(h, w, seed=1)
    p = tmp_path / "ours.exr"
    api.test_exr_write(p, img, normalized_by=0.5)
    out = C.POINTER(C.c_float)()
    ww, hh = C.c_int(), C.c_int()
    err = C.c_char_p()
    assert L.LoadEXR(C.byref(out), C.byref(ww), C.byref(hh), str(p).encode(), C.byref(err)) == 0, err.value
    try:
        assert (hh.value, ww.value) == (h, w)
        got = np.ctypeslib.as_array(out, shape=(h * w * 4,)).reshape(h, w, 4).copy()
    finally:
        C.CDLL(None).free(out)
    expect = img * np.float32(0.5)
    assert np.array_equal(got[..., :3].view(np.uint32), expect.view(np.uint32))
    assert np.all(got[..., 3] == 1.0)


@pytest.mark.parametrize("h,w", SIZES)
def test_reference_saved_exr_matches(built, tmp_path, h, w):
    """The reference's saveEXR path: RGBA, colours times the normalisation,
    alpha 1, written by tinyexr's SaveEXR(data, w, h, 4, fp16 = 0)."""
    L = tinyexr()
    img = image(h, w, seed=2)
    norm = np.float32(1 / 3)
    rgba = np.concatenate([img * norm, np.ones((h, w, 1), np.float32)], axis=-1)
    ref = tmp_path / "reference.exr"
    err = C.c_char_p()
    assert L.SaveEXR(np.ascontiguousarray(rgba).ctypes.data_as(C.POINTER(C.c_float)), w, h, 4, 0,
                     str(ref).encode(), C.byref(err)) == 0, err.value
    ours = tmp_path / "ours.exr"
    api.test_exr_write(ours, img, normalized_by=float(norm))
    a, ha = exr.read_exr(ref)
    b, hb = exr.read_exr(ours)
    for key in ("channels", "compression", "dataWindow", "displayWindow", "lineOrder"):
        assert ha[key] == hb[key], key
    for c in "ABGR":
        assert np.array_equal(a[c].view(np.uint32), b[c].view(np.uint32)), c


@pytest.mark.gpu
def test_film_save_exr(gpu_ctx, tmp_path):
    scene = api.Scene(gpu_ctx, SceneDesc(scenes.cornell(seed=1, envmap_exponent=7)))
    r = api.Renderer(scene, 40, 24)
    r.render(spp=8, max_depth=8)
    p = tmp_path / "frame.exr"
    r.save_exr(p)  # normalised by the samples
    raw = r.film()
    rgba = exr.read_rgba(p)
    assert np.array_equal(rgba[..., :3], raw * np.float32(1 / 8))
    assert np.allclose(rgba[..., :3], r.film(normalize=True), rtol=1e-6, atol=0)
    r.save_exr(p, normalized_by=2.0, compression="none")
    assert np.array_equal(exr.read_rgba(p)[..., :3], raw * np.float32(2.0))
