"""ctypes binding of the oracle library (oracle/oracle.h).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
# The same sources built with fused multiply-adds contracted (-ffp-contract=fast
# -mfma): every result may move by an ulp or so.  Rendering a scene with both
# measures how far the scene's own arithmetic amplifies rounding, the noise
# floor against which another implementation's per-sample match is judged.
LIB_FMA = HERE / "_build" / "liboracle_fma.so"


class OracleSettings(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32), ("max_depth", C.c_uint32),
                ("sampling_mode", C.c_uint32), ("rng", C.c_uint32), ("seed", C.c_uint64),
                ("first_sample", C.c_int64), ("threads", C.c_int32), ("film_fp64", C.c_int32),
                ("pixels", C.POINTER(C.c_uint32)), ("num_pixels", C.c_uint64)]


def build() -> Path:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_libs = {}


def fma_available() -> bool:
    """The contracted build needs a host CPU with FMA instructions."""
    try:
        return any(line.startswith("flags") and " fma " in line + " " for line in open("/proc/cpuinfo"))
    except OSError:
        return False


def lib(variant: str = ""):
    """The oracle library; variant "fma" is the contracted build (LIB_FMA)."""
    if variant not in _libs:
        path = {"": LIB, "fma": LIB_FMA}[variant]
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.oracle_scene_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
        L.oracle_scene_destroy.argtypes = [C.c_void_p]
        L.oracle_surface_emissive.argtypes = [C.c_void_p, C.POINTER(C.c_uint8)]
        L.oracle_scene_info.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32)]
        L.oracle_render.argtypes = [C.c_void_p, C.POINTER(OracleSettings), C.POINTER(C.c_double),
                                    C.POINTER(C.c_uint64)]
        L.oracle_prng.argtypes = [C.c_int32, C.c_uint64, C.c_uint64, C.c_int32, C.POINTER(C.c_float)]
        L.oracle_trace.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int32, C.c_int32, C.POINTER(C.c_float),
                                   C.POINTER(C.c_uint32)]
        L.oracle_fractal_noise3.argtypes = [C.POINTER(C.c_float), C.c_int32, C.c_float, C.c_float,
                                            C.POINTER(C.c_float)]
        L.oracle_material_eval.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_float), C.c_int32,
                                           C.POINTER(C.c_float)]
        L.oracle_scene_set_camera.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_sky_texture.argtypes = [C.c_int32, C.c_int32] + [C.c_float] * 5 + [C.POINTER(C.c_float)]
        L.oracle_sky_data.argtypes = [C.c_float, C.c_float, C.c_int32] + [C.c_float] * 5 + [C.POINTER(C.c_float)]
        L.oracle_normalize_image.argtypes = [C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_float, C.c_int32,
                                             C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]
        _libs[variant] = L
    return _libs[variant]


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


class OracleScene:
    def __init__(self, desc, variant: str = ""):
        """desc: raymond_b200._abi.SceneDesc; variant: "" or "fma" (see LIB_FMA)."""
        self.desc = desc
        self.L = lib(variant)
        self.h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = self.L.oracle_scene_create(C.byref(desc.c), C.byref(self.h), err, 512)
        if st != 0:
            raise RuntimeError(f"oracle_scene_create failed ({st}): {err.value.decode()}")

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.oracle_scene_destroy(self.h)
            self.h = C.c_void_p()

    def surface_emissive(self) -> np.ndarray:
        """Per surface material: 1 if it emits (a shape carrying it is a shape light)."""
        out = np.zeros(len(self.desc.scene["materials"]), np.uint8)
        self.L.oracle_surface_emissive(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    def set_camera(self, camera: dict) -> None:
        """Replace the camera (a camera dict as in the scene descriptions)."""
        from raymond_b200._abi import make_camera

        cam = make_camera(camera)
        if self.L.oracle_scene_set_camera(self.h, C.byref(cam)) != 0:
            raise RuntimeError("oracle_scene_set_camera failed")

    def info(self):
        t = C.c_uint64()
        n = C.c_int32()
        s = C.c_int32()
        self.L.oracle_scene_info(self.h, C.byref(t), C.byref(n), C.byref(s))
        return {"triangles": t.value, "lights": n.value, "shape_lights": s.value}

    def render(self, width, height, spp, max_depth, sampling_mode=2, rng=0, seed=1, first_sample=0, threads=0,
               film_fp64=False, pixels=None):
        """Film sums (H, W, 3) float64 and stats (paths, segments, shadow rays).
        `pixels`: trace only these linear pixel indices (y * width + x), with
        the full image's PRNG streams; the rest of the film stays zero."""
        st = OracleSettings(width, height, spp, max_depth, sampling_mode, rng, seed, first_sample, threads,
                            int(film_fp64))
        if pixels is not None:
            pixels = np.ascontiguousarray(pixels, np.uint32)
            st.pixels = pixels.ctypes.data_as(C.POINTER(C.c_uint32))
            st.num_pixels = len(pixels)
        film = np.zeros((height, width, 3), np.float64)
        stats = (C.c_uint64 * 3)()
        r = self.L.oracle_render(self.h, C.byref(st), film.ctypes.data_as(C.POINTER(C.c_double)), stats)
        if r != 0:
            raise RuntimeError(f"oracle_render failed ({r})")
        return film, {"paths": stats[0], "segments": stats[1], "shadow_rays": stats[2]}

    def trace(self, rays: np.ndarray, any_hit=False, exhaustive=False):
        """Closest hits (or occlusion with any_hit); `exhaustive` visits every
        box the ray enters instead of culling against the best hit so far."""
        rays = _f32(rays)
        n = len(rays)
        out = np.zeros((n, 4), np.float32)
        inst = np.zeros(n, np.uint32)
        mode = 1 if any_hit else 2 if exhaustive else 0
        self.L.oracle_trace(self.h, rays.ctypes.data_as(C.POINTER(C.c_float)), n, mode,
                           out.ctypes.data_as(C.POINTER(C.c_float)), inst.ctypes.data_as(C.POINTER(C.c_uint32)))
        return out, inst

    def material_eval(self, material: int, records: np.ndarray):
        records = _f32(records)
        n = len(records)
        out = np.zeros((n, 16), np.float32)
        r = self.L.oracle_material_eval(self.h, material, records.ctypes.data_as(C.POINTER(C.c_float)), n,
                                       out.ctypes.data_as(C.POINTER(C.c_float)))
        if r != 0:
            raise RuntimeError(f"oracle_material_eval failed ({r})")
        return out


def normalize_image(film: np.ndarray, exposure: float, accumulate: bool, frame_index: int,
                    tonemapping: int) -> np.ndarray:
    """normalizeImage restated: (h, w, 3 or 4) film sums -> (h, w, 4) float32."""
    film = np.asarray(film, np.float32)
    h, w = film.shape[:2]
    rgba = np.zeros((h, w, 4), np.float32)
    rgba[..., :3] = film[..., :3]
    out = np.zeros((h, w, 4), np.float32)
    lib().oracle_normalize_image(rgba.ctypes.data_as(C.POINTER(C.c_float)), w, h, exposure, int(accumulate),
                                 frame_index, tonemapping, out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def sky_texture(width: int, height: int, sun_elevation: float, altitude: float, air: float, dust: float,
                ozone: float) -> np.ndarray:
    """The Nishita sky texture restated: (height, width, 4) float32, XYZ in rgb."""
    out = np.zeros((height, width, 4), np.float32)
    lib().oracle_sky_texture(width, height, sun_elevation, altitude, air, dust, ozone,
                             out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def sky_data(sun_elevation, sun_rotation, sun_disc, sun_size, sun_intensity, altitude, air, dust) -> np.ndarray:
    """The TEX_SKY node's ten data values (sun disc colours, elevation, rotation, size or -1, intensity)."""
    out = np.zeros(10, np.float32)
    lib().oracle_sky_data(sun_elevation, sun_rotation, int(sun_disc), sun_size, sun_intensity, altitude, air, dust,
                          out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def prng(mode: int, a: int, b: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().oracle_prng(mode, a, b, n, out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def fractal_noise3(p: np.ndarray, detail: float, roughness: float) -> np.ndarray:
    p = _f32(p)
    out = np.zeros(len(p), np.float32)
    lib().oracle_fractal_noise3(p.ctypes.data_as(C.POINTER(C.c_float)), len(p), detail, roughness,
                                out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count() or 1
