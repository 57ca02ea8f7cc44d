"""ctypes binding of oracle/_ref/libref.so, the host build of the reference's
own device code (oracle/ref/Makefile).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parents[1] / "_ref" / "libref.so"
_fp = C.POINTER(C.c_float)
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        L.ref_prng_tea.argtypes = [C.c_uint32, C.c_uint32, C.c_int, _fp]
        L.ref_fractal_noise3.argtypes = [_fp, C.c_int, C.c_float, C.c_float, _fp]
        L.ref_num_materials.restype = C.c_int
        L.ref_material_eval.argtypes = [C.c_int, _fp, C.c_int, _fp]
        L.ref_material_eval.restype = C.c_int
        L.ref_set_texture.argtypes = [C.c_int, _fp, C.c_int, C.c_int]
        L.ref_set_texture.restype = C.c_int
        L.ref_scene_create.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_uint8)]
        L.ref_scene_create.restype = C.c_void_p
        L.ref_scene_destroy.argtypes = [C.c_void_p]
        L.ref_render.argtypes = [C.c_void_p] + [C.c_uint32] * 6 + [_fp]
        L.ref_render.restype = C.c_int
        L.ref_normalize_image.argtypes = [_fp, C.c_uint32, C.c_uint32, C.c_float] + [C.c_uint32] * 3 + [_fp]
        L.ref_normalize_image.restype = C.c_int
        _lib = L
    return _lib


def texels(img: np.ndarray) -> np.ndarray:
    """An image (h, w[, 1|3|4]) of uint8, uint16 or float32 as the RGBA floats a
    texture holds: integers normalised, one channel as (r, 0, 0, 1), RGB with alpha 1."""
    a = np.asarray(img)
    if a.ndim == 2:
        a = a[:, :, None]
    if a.dtype == np.uint8:
        f = a.astype(np.float32) / np.float32(255)
    elif a.dtype == np.uint16:
        f = a.astype(np.float32) / np.float32(65535)
    else:
        f = a.astype(np.float32)
    out = np.zeros(a.shape[:2] + (4,), np.float32)
    out[..., 3] = 1
    out[..., :a.shape[2]] = f
    return out


def set_textures(textures: dict) -> None:
    """Install the pinning scene's textures (in order) as the reference build's Context.textures."""
    for slot, img in enumerate(textures.values()):
        t = np.ascontiguousarray(texels(img))
        assert lib().ref_set_texture(slot, t.ctypes.data_as(_fp), t.shape[1], t.shape[0]) == 0


def set_texture(slot: int, rgba: np.ndarray) -> None:
    """Install one (h, w, 4) float texture at `slot` of the reference build's Context.textures."""
    t = np.ascontiguousarray(rgba, np.float32)
    assert lib().ref_set_texture(slot, t.ctypes.data_as(_fp), t.shape[1], t.shape[0]) == 0


def prng_tea(a: int, b: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().ref_prng_tea(a, b, n, out.ctypes.data_as(_fp))
    return out


def fractal_noise3(p: np.ndarray, detail: float, roughness: float) -> np.ndarray:
    p = np.ascontiguousarray(p, np.float32)
    out = np.zeros(len(p), np.float32)
    lib().ref_fractal_noise3(p.ctypes.data_as(_fp), len(p), detail, roughness, out.ctypes.data_as(_fp))
    return out


def material_eval(material: int, records: np.ndarray) -> np.ndarray:
    records = np.ascontiguousarray(records, np.float32)
    out = np.zeros((len(records), 16), np.float32)
    if lib().ref_material_eval(material, records.ctypes.data_as(_fp), len(records), out.ctypes.data_as(_fp)) != 0:
        raise ValueError(f"no material {material}")
    return out


def shading_records(n: int, seed: int) -> np.ndarray:
    """Random shading inputs in the record layout of ref_material_eval /
    oracle_material_eval: unit normals, wo in the normal's hemisphere."""
    rng = np.random.default_rng(seed)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    rec = np.zeros((n, 28), np.float32)
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
    rec[:, 24] = 1  # camera ray
    t = np.cross(nrm, unit(n))  # a tangent; the bitangent is normal x tangent
    rec[:, 25:28] = t / np.linalg.norm(t, axis=1, keepdims=True)
    return rec


class RefScene:
    """A scene set up for the reference's own kernels (host build).  `table`
    names its generated materials (pin_materials.ref_scenes); `emissive` is the
    per-surface-material emission flag (oracle_ctypes.OracleScene.surface_emissive)."""

    def __init__(self, desc, table: str, emissive: np.ndarray):
        self.desc = desc  # keeps the arrays the C structs point to alive
        self.emissive = np.ascontiguousarray(emissive, np.uint8)
        self.h = lib().ref_scene_create(C.byref(desc.c), table.encode(),
                                        self.emissive.ctypes.data_as(C.POINTER(C.c_uint8)))
        if not self.h:
            raise ValueError(f"no material table {table!r} in the reference build")

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_scene_destroy(self.h)
            self.h = None

    def render(self, width: int, height: int, frames: int, max_depth: int, sampling_mode: int = 2,
               first_frame: int = 0) -> np.ndarray:
        """Film (H, W, 4): rgb sums and write counts after `frames` one-sample frames."""
        film = np.zeros((height, width, 4), np.float32)
        lib().ref_render(self.h, width, height, frames, max_depth, sampling_mode, first_frame, film.ctypes.data_as(_fp))
        return film


def normalize_image(film: np.ndarray, exposure: float, accumulate: bool, frame_index: int,
                    tonemapping: int) -> np.ndarray:
    """The reference's normalizeImage kernel over a (h, w, 4) float32 film: (h, w, 4)."""
    film = np.ascontiguousarray(film, np.float32)
    h, w = film.shape[:2]
    out = np.zeros((h, w, 4), np.float32)
    lib().ref_normalize_image(film.ctypes.data_as(_fp), w, h, exposure, int(accumulate), frame_index, tonemapping,
                              out.ctypes.data_as(_fp))
    return out


SKY_LIB = Path(__file__).resolve().parents[1] / "_ref" / "libsky.so"


def sky_available() -> bool:
    return SKY_LIB.exists()


def sky_texture(width: int, height: int, sun_elevation: float, altitude: float, air: float, dust: float,
                ozone: float) -> np.ndarray:
    """The reference's SKY_nishita_skymodel_precompute_texture: (height, width, 3) XYZ (the stride-4
    buffer's fourth channel is never written by it)."""
    L = C.CDLL(str(SKY_LIB))
    L.SKY_nishita_skymodel_precompute_texture.argtypes = [_fp] + [C.c_int] * 5 + [C.c_float] * 5
    px = np.zeros((height, width, 4), np.float32)
    L.SKY_nishita_skymodel_precompute_texture(px.ctypes.data_as(_fp), 4, 0, height, width, height, sun_elevation,
                                              altitude, air, dust, ozone)
    return px[..., :3]


def sky_sun(sun_elevation: float, angular_diameter: float, altitude: float, air: float, dust: float) -> np.ndarray:
    """The reference's SKY_nishita_skymodel_precompute_sun: bottom and top XYZ (6 floats)."""
    L = C.CDLL(str(SKY_LIB))
    L.SKY_nishita_skymodel_precompute_sun.argtypes = [C.c_float] * 5 + [_fp, _fp]
    out = np.zeros(6, np.float32)
    L.SKY_nishita_skymodel_precompute_sun(sun_elevation, angular_diameter, altitude, air, dust,
                                          out[:3].ctypes.data_as(_fp), out[3:].ctypes.data_as(_fp))
    return out
