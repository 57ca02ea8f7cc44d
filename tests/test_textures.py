"""Image textures (the TexImage / TexEnvironment nodes): image files, scene
files that carry textures, and the code generated for the nodes.

The sampling itself is checked on the GPU against the oracle
(test_parity_gpu.py) and, for the node around it, the oracle against the
reference's own node library (test_ref_pin.py, the `image_textures` pinning
material).
"""
import ctypes as C
import struct
import sys
import warnings
import zlib
from pathlib import Path

import numpy as np
import pytest

from raymond_b200 import api, exr, loader, png, scenes
from raymond_b200._abi import SceneDesc

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle" / "ref"))
import pin_materials  # noqa: E402

TINYEXR = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libtinyexr.so"


@pytest.mark.parametrize("shape,dtype", [((7, 5), np.uint8), ((6, 9, 3), np.uint8), ((5, 4, 4), np.uint8),
                                         ((8, 3), np.uint16), ((4, 6, 4), np.uint16), ((33, 17, 3), np.uint8)])
@pytest.mark.parametrize("filters", [(0,), (1,), (2,), (3,), (4,), (0, 1, 2, 3, 4)])
def test_png_round_trip(tmp_path, shape, dtype, filters):
    img = np.random.default_rng(len(shape) + shape[0]).integers(0, np.iinfo(dtype).max + 1, shape, dtype=dtype)
    png.write_png(tmp_path / "a.png", img, filters=filters)
    back = png.read_png(tmp_path / "a.png")
    assert back.dtype == dtype
    assert np.array_equal(back, img if img.ndim == 3 else img[:, :, None])


def _chunk(kind, body):
    return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)


def test_png_palette_and_grey_alpha(tmp_path):
    pal = np.array([[10, 20, 30], [200, 100, 50], [0, 255, 7]], np.uint8)
    idx = np.array([[0, 1, 2], [2, 1, 0]], np.uint8)
    raw = b"".join(b"\0" + r.tobytes() for r in idx)
    data = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", 3, 2, 8, 3, 0, 0, 0)) + \
        _chunk(b"PLTE", pal.tobytes()) + _chunk(b"tRNS", bytes([255, 128])) + \
        _chunk(b"IDAT", zlib.compress(raw)) + _chunk(b"IEND", b"")
    (tmp_path / "p.png").write_bytes(data)
    got = png.read_png(tmp_path / "p.png")
    assert np.array_equal(got[..., :3], pal[idx])
    assert np.array_equal(got[..., 3], np.array([255, 128, 255], np.uint8)[idx])
    ga = np.stack([np.arange(6, dtype=np.uint8).reshape(2, 3), np.full((2, 3), 9, np.uint8)], -1)
    raw = b"".join(b"\0" + r.tobytes() for r in ga.reshape(2, -1))
    data = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", 3, 2, 8, 4, 0, 0, 0)) + \
        _chunk(b"IDAT", zlib.compress(raw)) + _chunk(b"IEND", b"")
    (tmp_path / "g.png").write_bytes(data)
    got = png.read_png(tmp_path / "g.png")
    assert np.array_equal(got, np.stack([ga[..., 0]] * 3 + [ga[..., 1]], -1))
    with pytest.raises(png.PngError):
        png.read_png(_bad(tmp_path))


def _bad(tmp_path):
    p = tmp_path / "bad.png"
    p.write_bytes(b"not a png at all")
    return p


def test_exr_writer_loads_in_reference_library(built, tmp_path):
    img = np.random.default_rng(3).exponential(1.0, (5, 7, 3)).astype(np.float32)
    exr.write_exr(tmp_path / "a.exr", img)
    assert np.array_equal(exr.read_rgba(tmp_path / "a.exr")[..., :3], img)
    assert np.array_equal(loader.read_image(tmp_path / "a.exr"), img)
    if not TINYEXR.exists():
        pytest.skip("oracle/_ref/libtinyexr.so not built")
    L = C.CDLL(str(TINYEXR))
    out = C.POINTER(C.c_float)()
    w, h, err = C.c_int(), C.c_int(), C.c_char_p()
    assert L.LoadEXR(C.byref(out), C.byref(w), C.byref(h), str(tmp_path / "a.exr").encode(), C.byref(err)) == 0
    got = np.ctypeslib.as_array(out, shape=(35 * 4,)).reshape(5, 7, 4).copy()
    C.CDLL(None).free(out)
    assert np.array_equal(got[..., :3], img)


def test_scene_file_with_textures_round_trip(built, tmp_path):
    sc = pin_materials.scene()
    path = tmp_path / "scene.json"
    loader.save_scene(sc, path)
    assert (tmp_path / "textures" / "albedo.png").exists() and (tmp_path / "textures" / "sky.exr").exists()
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        back, _ = loader.load_scene(path)
    # the node naming a file that was never exported is reported and left out
    assert any("not_exported.jpg" in str(x.message) for x in w)
    assert set(back["textures"]) == set(sc["textures"])
    for name, img in sc["textures"].items():
        want = img if img.ndim == 3 else img[:, :, None]
        assert back["textures"][name].dtype == img.dtype
        assert np.array_equal(back["textures"][name], want), name


def test_codegen_texture_nodes(built):
    src = api.generate_source(pin_materials.scene(), hoist=False)
    assert ("TexImage<0, kTexImage::INTERPOLATION_LINEAR, kTexImage::PROJECTION_FLAT, kTexImage::EXTENSION_REPEAT, "
            "kTexImage::ALPHA_STRAIGHT, kTexImage::COLOR_SPACE_SRGB, kTexImage::PIXEL_FORMAT_RGBA>") in src
    assert "TexImage<1, kTexImage::INTERPOLATION_LINEAR, kTexImage::PROJECTION_FLAT" in src
    assert "kTexImage::COLOR_SPACE_NON_COLOR, kTexImage::PIXEL_FORMAT_R>" in src
    assert "TexImage<2, kTexImage::INTERPOLATION_LINEAR, kTexImage::PROJECTION_EQUIRECTANGULAR" in src
    assert "kTexImage::COLOR_SPACE_XYZ, kTexImage::PIXEL_FORMAT_RGBA>" in src
    # the sky material's generated texture follows the scene's three images
    assert "TexNishita<3>" in src
    # the missing file: the zero texture after them, single channel
    assert "TexImage<4, kTexImage::INTERPOLATION_LINEAR, kTexImage::PROJECTION_FLAT" in src
    # the reference's node knows linear interpolation only
    sc = pin_materials.scene()
    graph = dict(sc["materials"])["image_textures"]
    graph["Albedo"]["parameters"]["interpolation"] = "Closest"
    with pytest.raises(api.RmdError):
        api.generate_source(sc)


def test_texture_nodes_compile(built):
    n, _ = api.jit_compile(pin_materials.scene())
    assert n > 0


def test_invalid_textures_rejected(built):
    sc = scenes.cornell(seed=1, envmap_exponent=4)
    sc["textures"] = {"bad.png": np.zeros((4, 4, 2), np.uint8)}
    with pytest.raises(ValueError):
        SceneDesc(sc)
