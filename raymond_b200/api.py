"""Python host API over the C ABI of librmd.so.

Mirrors the reference's host objects: `Scene` is SceneLoader.loadScene's
result (SceneLoader.swift:46-143), `Renderer` is Renderer
(Renderer.swift:270-808) with render() = execute(in:) repeated `spp` times,
set_size / reset / set_camera, film read-out with normalizeImage's
arithmetic, and per-stage statistics (RendererCounters).

Every call goes through librmd.so; there is no Python or CPU fallback: when
the library or a GPU is missing the calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Any

import numpy as np

from . import _abi
from ._abi import RenderSettings, SceneDesc, Stats

LIB_PATH = Path(__file__).resolve().parent / "librmd.so"

# every function the C headers declare (include/raymond.h, include/raymond_testing.h)
EXPORTS = [
    "rmd_last_error", "rmd_version", "rmd_context_create", "rmd_context_destroy", "rmd_scene_create",
    "rmd_scene_destroy", "rmd_scene_info", "rmd_renderer_create", "rmd_renderer_destroy", "rmd_renderer_set_size",
    "rmd_renderer_reset", "rmd_renderer_set_camera", "rmd_render", "rmd_film_read", "rmd_film_read_f64",
    "rmd_film_samples", "rmd_renderer_stats", "rmd_render_noalloc", "rmd_renderer_autotune",
    "rmd_renderer_set_tuning", "rmd_renderer_set_guide", "rmd_renderer_guide_stats", "rmd_guide_param_count",
    "rmd_renderer_guide_params", "rmd_batch_create", "rmd_batch_destroy", "rmd_batch_reset", "rmd_batch_render",
    "rmd_batch_film_read", "rmd_batch_film_read_f64", "rmd_batch_stats", "rmd_batch_autotune",
    "rmd_batch_set_guide", "rmd_batch_guide_stats", "rmd_context_set_bvh_builder", "rmd_scene_bvh_stats",
    "rmd_film_save_exr", "rmd_batch_film_save_exr", "rmd_scene_instance_data", "rmd_render_frame",
    "rmd_film_normalize", "rmd_film_device", "rmd_film_set_samples",
    "rmd_test_prng", "rmd_test_trace", "rmd_test_material_eval", "rmd_test_generate_source", "rmd_test_jit_compile",
    "rmd_test_guide_forward", "rmd_test_guide_gradient", "rmd_test_guide_mixture", "rmd_test_bvh_read",
    "rmd_test_exr_write", "rmd_test_guide_adam",
]


class RmdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """Load librmd.so (build it first with raymond_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m raymond_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    P = C.POINTER
    sig = {
        "rmd_last_error": ([], C.c_char_p),
        "rmd_version": ([], C.c_char_p),
        "rmd_context_create": ([C.c_int32, P(vp)], C.c_int32),
        "rmd_context_set_bvh_builder": ([vp, C.c_uint32], C.c_int32),
        "rmd_scene_bvh_stats": ([vp, P(_abi.BvhStats)], C.c_int32),
        "rmd_test_bvh_read": ([vp, vp, C.c_uint64, P(C.c_float), C.c_uint64], C.c_int32),
        "rmd_film_save_exr": ([vp, C.c_char_p, C.c_float, C.c_uint32], C.c_int32),
        "rmd_batch_film_save_exr": ([vp, C.c_int32, C.c_char_p, C.c_float, C.c_uint32], C.c_int32),
        "rmd_test_exr_write": ([C.c_char_p, P(C.c_float), C.c_int32, C.c_int32, C.c_float, C.c_uint32], C.c_int32),
        "rmd_context_destroy": ([vp], None),
        "rmd_scene_create": ([vp, P(_abi.SceneDescC), P(vp)], C.c_int32),
        "rmd_scene_destroy": ([vp], None),
        "rmd_scene_info": ([vp, P(C.c_uint64), P(C.c_uint64), P(C.c_int32)], C.c_int32),
        "rmd_scene_instance_data": ([vp, P(_abi.PerInstanceData), C.c_int32, P(C.c_int32)], C.c_int32),
        "rmd_render_frame": ([vp, P(_abi.Uniforms), C.c_uint32], C.c_int32),
        "rmd_film_normalize": ([vp, P(_abi.Uniforms), P(C.c_float)], C.c_int32),
        "rmd_renderer_create": ([vp, C.c_uint32, C.c_uint32, C.c_uint32, P(vp)], C.c_int32),
        "rmd_renderer_destroy": ([vp], None),
        "rmd_renderer_set_size": ([vp, C.c_uint32, C.c_uint32], C.c_int32),
        "rmd_renderer_reset": ([vp], C.c_int32),
        "rmd_renderer_set_camera": ([vp, P(_abi.Camera)], C.c_int32),
        "rmd_render": ([vp, P(RenderSettings)], C.c_int32),
        "rmd_film_read": ([vp, P(C.c_float), C.c_int32, C.c_uint32, C.c_float], C.c_int32),
        "rmd_film_read_f64": ([vp, P(C.c_double)], C.c_int32),
        "rmd_film_samples": ([vp, P(C.c_uint64)], C.c_int32),
        "rmd_film_device": ([vp, P(vp), P(C.c_uint64)], C.c_int32),
        "rmd_film_set_samples": ([vp, C.c_uint64], C.c_int32),
        "rmd_renderer_stats": ([vp, P(Stats)], C.c_int32),
        "rmd_renderer_autotune": ([vp, P(RenderSettings), P(_abi.TuneResult)], C.c_int32),
        "rmd_renderer_set_tuning": ([vp, P(_abi.TuneResult)], C.c_int32),
        "rmd_renderer_set_guide": ([vp, P(_abi.GuideSettings)], C.c_int32),
        "rmd_renderer_guide_stats": ([vp, P(_abi.GuideStats)], C.c_int32),
        "rmd_guide_param_count": ([], C.c_int32),
        "rmd_renderer_guide_params": ([vp, P(C.c_float), C.c_int32], C.c_int32),
        "rmd_test_guide_forward": ([P(C.c_float), P(C.c_float), C.c_int32, P(C.c_float)], C.c_int32),
        "rmd_test_guide_gradient": ([P(C.c_float), P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float)], C.c_int32),
        "rmd_test_guide_mixture": ([P(C.c_float), P(C.c_float), C.c_int32, P(C.c_float), P(C.c_float), C.c_int32,
                                    P(C.c_float)], C.c_int32),
        "rmd_batch_create": ([vp, P(_abi.SceneDescC), C.c_int32, P(_abi.BatchView), C.c_int32, C.c_uint32, C.c_uint32,
                              P(vp)], C.c_int32),
        "rmd_batch_destroy": ([vp], None),
        "rmd_batch_reset": ([vp], C.c_int32),
        "rmd_batch_render": ([vp, P(RenderSettings)], C.c_int32),
        "rmd_batch_film_read": ([vp, C.c_int32, P(C.c_float), C.c_int32, C.c_uint32, C.c_float], C.c_int32),
        "rmd_batch_film_read_f64": ([vp, C.c_int32, P(C.c_double)], C.c_int32),
        "rmd_batch_stats": ([vp, P(Stats)], C.c_int32),
        "rmd_batch_autotune": ([vp, P(RenderSettings), P(_abi.TuneResult)], C.c_int32),
        "rmd_batch_set_guide": ([vp, P(_abi.GuideSettings)], C.c_int32),
        "rmd_batch_guide_stats": ([vp, P(_abi.GuideStats)], C.c_int32),
        "rmd_render_noalloc": ([vp, P(_abi.Camera), C.c_uint32, C.c_uint32, P(RenderSettings), C.c_void_p,
                                C.c_uint32], C.c_int32),
        "rmd_test_guide_adam": ([P(C.c_float)] * 4 + [C.c_int32, C.c_float] + [P(C.c_float)] * 3 + [P(C.c_uint16)],
                                C.c_int32),
        "rmd_test_prng": ([C.c_uint32, C.c_uint64, C.c_uint64, C.c_int32, P(C.c_float)], C.c_int32),
        "rmd_test_trace": ([vp, P(C.c_float), C.c_int32, C.c_int32, P(C.c_float), P(C.c_uint32)], C.c_int32),
        "rmd_test_material_eval": ([vp, C.c_int32, P(C.c_float), C.c_int32, P(C.c_float)], C.c_int32),
        "rmd_test_generate_source": ([P(_abi.SceneDescC), C.c_int32, C.c_char_p, C.c_int64, P(C.c_int64)], C.c_int32),
        "rmd_test_jit_compile": ([P(_abi.SceneDescC), C.c_int32, C.c_char_p, C.c_int64, P(C.c_int64)], C.c_int32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != 0:
        raise RmdError(status, lib().rmd_last_error().decode(errors="replace"))


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Context:
    """A CUDA device and stream (rmd_context).  `bvh_builder`: "host" (binned
    SAH on the host) or "gpu" (built on the device) for the scenes created
    in this context."""

    def __init__(self, device: int = 0, bvh_builder: str = "host"):
        self.device = device
        self.h = C.c_void_p()
        check(lib().rmd_context_create(device, C.byref(self.h)))
        self.set_bvh_builder(bvh_builder)

    def set_bvh_builder(self, builder: str) -> None:
        if builder not in _abi.BVH_BUILDERS:
            raise ValueError(f"bvh_builder must be one of {sorted(_abi.BVH_BUILDERS)}, not {builder!r}")
        check(lib().rmd_context_set_bvh_builder(self.h, _abi.BVH_BUILDERS[builder]))

    def close(self):
        if self.h.value:
            lib().rmd_context_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Geometry, BVH, JIT-compiled materials and lights on one device."""

    def __init__(self, ctx: Context, scene: dict[str, Any] | SceneDesc):
        self.ctx = ctx
        self.desc = scene if isinstance(scene, SceneDesc) else SceneDesc(scene)
        self.h = C.c_void_p()
        check(lib().rmd_scene_create(ctx.h, C.byref(self.desc.c), C.byref(self.h)))

    def info(self) -> dict[str, int]:
        t, n = C.c_uint64(), C.c_uint64()
        lights = C.c_int32()
        check(lib().rmd_scene_info(self.h, C.byref(t), C.byref(n), C.byref(lights)))
        return {"triangles": t.value, "bvh_nodes": n.value, "lights": lights.value}

    def bvh_stats(self) -> dict[str, float]:
        """Builder, levels, nodes, build time (ms) and surface-area cost of the BVH."""
        st = _abi.BvhStats()
        check(lib().rmd_scene_bvh_stats(self.h, C.byref(st)))
        names = {v: k for k, v in _abi.BVH_BUILDERS.items()}
        return {"builder": names.get(st.builder, st.builder), "levels": st.levels, "nodes": st.nodes,
                "build_ms": st.build_ms, "sah_cost": st.sah_cost, "cluster_iterations": st.cluster_iterations}

    def bvh_arrays(self) -> tuple[np.ndarray, np.ndarray]:
        """The BVH as the traversal kernels read it (test hook): 80-byte nodes
        as a (nodes, 80) uint8 array and the leaf-ordered triangles (n, 12) float32."""
        info = self.info()
        nodes = np.zeros((max(1, info["bvh_nodes"]), 80), np.uint8)
        tris = np.zeros((max(1, info["triangles"]), 12), np.float32)
        check(lib().rmd_test_bvh_read(self.h, nodes.ctypes.data_as(C.c_void_p), nodes.shape[0], _f32p(tris),
                                      tris.shape[0]))
        return nodes[:info["bvh_nodes"]], tris[:info["triangles"]]

    def instance_data(self) -> list[_abi.PerInstanceData]:
        """The per-instance records (bridge/PerInstanceData.hpp layout), one per entity."""
        n = C.c_int32()
        check(lib().rmd_scene_instance_data(self.h, None, 0, C.byref(n)))
        arr = (_abi.PerInstanceData * max(1, n.value))()
        check(lib().rmd_scene_instance_data(self.h, arr, n.value, C.byref(n)))
        return list(arr)[:n.value]

    def trace(self, rays: np.ndarray, any_hit: bool = False):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        out = np.zeros((n, 4), np.float32)
        inst = np.zeros(n, np.uint32)
        check(lib().rmd_test_trace(self.h, _f32p(rays), n, int(any_hit), _f32p(out),
                                   inst.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out, inst

    def material_eval(self, material: int, records: np.ndarray) -> np.ndarray:
        records = np.ascontiguousarray(records, np.float32)
        out = np.zeros((len(records), 16), np.float32)
        check(lib().rmd_test_material_eval(self.h, material, _f32p(records), len(records), _f32p(out)))
        return out

    def close(self):
        if self.h.value:
            lib().rmd_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceFilm:
    """A renderer's device film seen through the CUDA array interface (no copy)."""

    def __init__(self, ptr: int, shape: tuple[int, int, int]):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


class Renderer:
    """Wavefront renderer for one film (rmd_renderer)."""

    def __init__(self, scene: Scene, width: int, height: int, pool_size: int = 0):
        self.scene = scene
        self.width, self.height = width, height
        self.h = C.c_void_p()
        check(lib().rmd_renderer_create(scene.h, width, height, pool_size, C.byref(self.h)))

    def render(self, spp: int, max_depth: int = 8, sampling_mode: int = _abi.SAMPLING_MIS, rng: int = _abi.RNG_PCG32,
               seed: int = 1, first_sample: int = -1, film_fp64: bool = False) -> None:
        s = RenderSettings(spp, max_depth, sampling_mode, rng, seed, first_sample, int(film_fp64), 0)
        check(lib().rmd_render(self.h, C.byref(s)))

    def film(self, normalize: bool = False, tonemapping: int = _abi.TONEMAP_LINEAR, exposure: float = 1.0,
             out: np.ndarray | None = None) -> np.ndarray:
        """The film (H, W, 3) float32 (rmd_film_read); `out`: a C-contiguous float32
        array of that shape to read into (e.g. in pinned host memory)."""
        if out is None:
            out = np.zeros((self.height, self.width, 3), np.float32)
        elif out.shape != (self.height, self.width, 3) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape (height, width, 3)")
        check(lib().rmd_film_read(self.h, _f32p(out), int(normalize), tonemapping, exposure))
        return out

    def film_device(self) -> "DeviceFilm":
        """The film in device memory, zero-copy (rmd_film_device): an object with
        __cuda_array_interface__ of shape (H, W, 4) float32 (RGB sums, path count),
        e.g. for torch.as_tensor(..., device="cuda") and a collective."""
        ptr = C.c_void_p()
        n = C.c_uint64()
        check(lib().rmd_film_device(self.h, C.byref(ptr), C.byref(n)))
        return DeviceFilm(ptr.value, (self.height, self.width, 4))

    def film_tensor(self):
        """The device film as a torch CUDA tensor (H, W, 4) aliasing the library's buffer."""
        import torch

        return torch.as_tensor(self.film_device(), device=f"cuda:{self.scene.ctx.device}")

    def set_samples(self, samples: int) -> None:
        """The film's sample count after other renderers' films were summed into it."""
        check(lib().rmd_film_set_samples(self.h, samples))

    def render_frame(self, uniforms: _abi.Uniforms, max_depth: int = 8) -> None:
        """One frame of the reference's Renderer.execute driven by its Uniforms (rmd_render_frame)."""
        check(lib().rmd_render_frame(self.h, C.byref(uniforms), max_depth))

    def film_normalize(self, uniforms: _abi.Uniforms) -> np.ndarray:
        """normalizeImage with the reference's Uniforms (rmd_film_normalize): (H, W, 4) float32."""
        out = np.zeros((self.height, self.width, 4), np.float32)
        check(lib().rmd_film_normalize(self.h, C.byref(uniforms), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def film64(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 3), np.float64)
        check(lib().rmd_film_read_f64(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def save_exr(self, path, normalized_by: float = 0.0, compression: str = "auto") -> None:
        """The film as an OpenEXR file (rmd_film_save_exr): RGBA float32, colours
        times `normalized_by` (0: divided by the samples)."""
        check(lib().rmd_film_save_exr(self.h, str(path).encode(), normalized_by, _exr_compression(compression)))

    def samples(self) -> int:
        v = C.c_uint64()
        check(lib().rmd_film_samples(self.h, C.byref(v)))
        return v.value

    def reset(self) -> None:
        check(lib().rmd_renderer_reset(self.h))

    def set_size(self, width: int, height: int) -> None:
        check(lib().rmd_renderer_set_size(self.h, width, height))
        self.width, self.height = width, height

    def set_camera(self, camera: dict[str, Any]) -> None:
        cam = _abi.make_camera(camera)
        check(lib().rmd_renderer_set_camera(self.h, C.byref(cam)))

    def autotune(self, spp: int = 64, max_depth: int = 8, sampling_mode: int = _abi.SAMPLING_MIS,
                 rng: int = _abi.RNG_PCG32, seed: int = 1) -> dict[str, float]:
        """Pick launch choices with short calibration renders (clears the film)."""
        s = RenderSettings(spp, max_depth, sampling_mode, rng, seed, -1, 0, 0)
        res = _abi.TuneResult()
        check(lib().rmd_renderer_autotune(self.h, C.byref(s), C.byref(res)))
        return {k: getattr(res, k) for k, _ in _abi.TuneResult._fields_}

    def set_tuning(self, tuning: dict[str, float]) -> None:
        """Apply launch choices returned by autotune() (here or in another process)."""
        t = _abi.TuneResult(**{k: tuning.get(k, 0) for k, _ in _abi.TuneResult._fields_})
        check(lib().rmd_renderer_set_tuning(self.h, C.byref(t)))

    def stats(self) -> dict[str, float]:
        s = Stats()
        check(lib().rmd_renderer_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def set_guide(self, sampling: bool = True, training: bool = True, batch_size: int = 0,
                  learning_rate: float = 0.0, reset: bool = False, seed: int = 0, step_records: int = 0,
                  replay_records: int = 0, steps_per_batch: int = 0, light_records: bool = True,
                  guided_depth: int = 0) -> None:
        """Learned path guiding (rmd_renderer_set_guide): sample directions from
        the guide mixture by one-sample MIS and/or train the network online
        during render().  One Adam step per `batch_size` tracer samples (0 =
        2^20), learning rate 0 = 1e-3, each step on `step_records` records
        (0 = 2^13) drawn from a ring of the latest `replay_records` (0 = 2^18);
        `steps_per_batch` (0 = 8) Adam steps per batch; `light_records`: the
        light samples of every vertex are training samples too; vertices of
        path depth below `guided_depth` (0 = all) sample from the guide.  The
        network is initialised from `seed` on first use or when `reset` is set."""
        g = _abi.GuideSettings(int(sampling), int(training), batch_size, learning_rate, int(reset), seed,
                               step_records, replay_records, steps_per_batch, int(not light_records), guided_depth)
        check(lib().rmd_renderer_set_guide(self.h, C.byref(g)))

    def guide_stats(self) -> dict[str, float]:
        g = _abi.GuideStats()
        check(lib().rmd_renderer_guide_stats(self.h, C.byref(g)))
        return {k: getattr(g, k) for k, _ in _abi.GuideStats._fields_ if k != "reserved"}

    def guide_params(self) -> np.ndarray:
        """The guide network's FP32 parameters (layout of rmd_renderer_guide_params)."""
        out = np.zeros(guide_param_count(), np.float32)
        check(lib().rmd_renderer_guide_params(self.h, _f32p(out), 0))
        return out

    def set_guide_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.size != guide_param_count():
            raise ValueError(f"expected {guide_param_count()} parameters, got {p.size}")
        check(lib().rmd_renderer_guide_params(self.h, _f32p(p), 1))

    def close(self):
        if self.h.value:
            lib().rmd_renderer_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many scenes and views traced by one wavefront and one CUDA-graph
    launch (rmd_batch): `views` is a list of dicts {scene: index into
    `scenes`, width, height, camera (optional; the scene's camera)}."""

    def __init__(self, ctx: Context, scenes: list, views: list[dict[str, Any]], pool_size: int = 0,
                 graph: bool = True):
        self.ctx = ctx
        self.descs = [s if isinstance(s, SceneDesc) else SceneDesc(s) for s in scenes]
        arr = (_abi.SceneDescC * len(self.descs))(*[d.c for d in self.descs])
        self._arr = arr
        vs = (_abi.BatchView * len(views))()
        self.sizes = []
        for i, v in enumerate(views):
            known = 0 <= v["scene"] < len(self.descs)  # an unknown index is the library's to reject
            cam = v.get("camera") or self.descs[v["scene"] if known else 0].scene["camera"]
            vs[i] = _abi.BatchView(scene=v["scene"], width=v["width"], height=v["height"], camera=_abi.make_camera(cam))
            self.sizes.append((v["height"], v["width"]))
        self.h = C.c_void_p()
        flags = 0 if graph else _abi.BATCH_NO_GRAPH
        check(lib().rmd_batch_create(ctx.h, arr, len(self.descs), vs, len(views), pool_size, flags,
                                     C.byref(self.h)))

    def render(self, spp: int, max_depth: int = 8, sampling_mode: int = _abi.SAMPLING_MIS, rng: int = _abi.RNG_PCG32,
               seed: int = 1, first_sample: int = -1, film_fp64: bool = False) -> None:
        s = RenderSettings(spp, max_depth, sampling_mode, rng, seed, first_sample, int(film_fp64), 0)
        check(lib().rmd_batch_render(self.h, C.byref(s)))

    def film(self, view: int, normalize: bool = False, tonemapping: int = _abi.TONEMAP_LINEAR,
             exposure: float = 1.0) -> np.ndarray:
        h, w = self.sizes[view]
        out = np.zeros((h, w, 3), np.float32)
        check(lib().rmd_batch_film_read(self.h, view, _f32p(out), int(normalize), tonemapping, exposure))
        return out

    def film64(self, view: int) -> np.ndarray:
        h, w = self.sizes[view]
        out = np.zeros((h, w, 3), np.float64)
        check(lib().rmd_batch_film_read_f64(self.h, view, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def save_exr(self, view: int, path, normalized_by: float = 0.0, compression: str = "auto") -> None:
        check(lib().rmd_batch_film_save_exr(self.h, view, str(path).encode(), normalized_by,
                                            _exr_compression(compression)))

    def reset(self) -> None:
        check(lib().rmd_batch_reset(self.h))

    def stats(self) -> dict[str, float]:
        s = Stats()
        check(lib().rmd_batch_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def autotune(self, spp: int = 32, max_depth: int = 10, sampling_mode: int = _abi.SAMPLING_MIS,
                 rng: int = _abi.RNG_PCG32, seed: int = 1) -> dict[str, float]:
        s = RenderSettings(spp, max_depth, sampling_mode, rng, seed, -1, 0, 0)
        res = _abi.TuneResult()
        check(lib().rmd_batch_autotune(self.h, C.byref(s), C.byref(res)))
        return {k: getattr(res, k) for k, _ in _abi.TuneResult._fields_}

    def set_guide(self, sampling: bool = True, training: bool = True, batch_size: int = 0,
                  learning_rate: float = 0.0, reset: bool = False, seed: int = 0, step_records: int = 0,
                  replay_records: int = 0, steps_per_batch: int = 0, light_records: bool = True,
                  guided_depth: int = 0) -> None:
        """Learned path guiding for a batch whose views all show one scene
        (same settings as Renderer.set_guide)."""
        g = _abi.GuideSettings(int(sampling), int(training), batch_size, learning_rate, int(reset), seed,
                               step_records, replay_records, steps_per_batch, int(not light_records), guided_depth)
        check(lib().rmd_batch_set_guide(self.h, C.byref(g)))

    def guide_stats(self) -> dict[str, float]:
        g = _abi.GuideStats()
        check(lib().rmd_batch_guide_stats(self.h, C.byref(g)))
        return {k: getattr(g, k) for k, _ in _abi.GuideStats._fields_ if k != "reserved"}

    def close(self):
        if self.h.value:
            lib().rmd_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_noalloc(scene: Scene, camera: dict[str, Any], width: int, height: int, film_device_ptr: int, spp: int,
                   first_sample: int, max_depth: int = 8, sampling_mode: int = _abi.SAMPLING_MIS,
                   rng: int = _abi.RNG_PCG32, seed: int = 1, pool_size: int = 0) -> None:
    """rmd_render_noalloc: adds `spp` samples to a caller-owned device film of
    width*height float4 (RGB sums, path count) without allocating memory."""
    cam = _abi.make_camera(camera)
    s = RenderSettings(spp, max_depth, sampling_mode, rng, seed, first_sample, 0, 0)
    check(lib().rmd_render_noalloc(scene.h, C.byref(cam), width, height, C.byref(s), C.c_void_p(film_device_ptr),
                                   pool_size))


def load_scene(ctx: "Context", path) -> tuple["Scene", tuple[int, int] | None]:
    """A scene from the reference's on-disk format (exporter JSON + PLY meshes,
    raymond_b200.loader) and the file's render resolution."""
    from . import loader

    sc, size = loader.load_scene(path)
    return Scene(ctx, sc), size


def guide_param_count() -> int:
    return int(lib().rmd_guide_param_count())


def guide_forward(params: np.ndarray, features: np.ndarray) -> np.ndarray:
    """Test hook: the guide network's raw outputs (n, 48) for explicit features (n, 7)."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(features, np.float32).reshape(-1, 7)
    out = np.zeros((f.shape[0], 48), np.float32)
    check(lib().rmd_test_guide_forward(_f32p(p), _f32p(f), f.shape[0], _f32p(out)))
    return out


def guide_gradient(params: np.ndarray, records: np.ndarray) -> tuple[np.ndarray, float]:
    """Test hook: gradient of the mean training loss over `records` (n, 12:
    features 7, direction 3, BSDF pdf, target) and the loss itself."""
    p = np.ascontiguousarray(params, np.float32)
    r = np.ascontiguousarray(records, np.float32).reshape(-1, 12)
    grad = np.zeros(p.size, np.float32)
    loss = C.c_float()
    check(lib().rmd_test_guide_gradient(_f32p(p), _f32p(r), r.shape[0], _f32p(grad), C.byref(loss)))
    return grad, loss.value


def guide_adam(params: np.ndarray, grad: np.ndarray, m: np.ndarray, v: np.ndarray, step: int, lr: float):
    """Test hook: one Adam step on the device: (params, m, v, bf16 weight bits)."""
    f = [np.ascontiguousarray(a, np.float32) for a in (params, grad, m, v)]
    outs = [np.zeros_like(f[0]) for _ in range(3)]
    bits = np.zeros(guide_param_count(), np.uint16)  # the first (weights) entries are written
    check(lib().rmd_test_guide_adam(*[_f32p(a) for a in f], step, lr, *[_f32p(a) for a in outs],
                                    bits.ctypes.data_as(C.POINTER(C.c_uint16))))
    return outs[0], outs[1], outs[2], bits


def guide_mixture(outputs: np.ndarray, u: np.ndarray, queries: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Test hook: decode one output vector (48) into the packed mixture, draw a
    direction per row of u (n, 3) with its pdf (n, 4), and evaluate the pdf at
    queries (m, 3)."""
    o = np.ascontiguousarray(outputs, np.float32).reshape(48)
    uu = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 3)
    dp = np.zeros((uu.shape[0], 4), np.float32)
    pdf = np.zeros(q.shape[0], np.float32)
    check(lib().rmd_test_guide_mixture(_f32p(o), _f32p(uu), uu.shape[0], _f32p(dp), _f32p(q), q.shape[0], _f32p(pdf)))
    return dp, pdf


def generate_source(scene: dict[str, Any] | SceneDesc, hoist: bool = True) -> str:
    """The CUDA source the material JIT emits for a scene (no GPU needed)."""
    desc = scene if isinstance(scene, SceneDesc) else SceneDesc(scene)
    need = C.c_int64()
    check(lib().rmd_test_generate_source(C.byref(desc.c), int(hoist), None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(lib().rmd_test_generate_source(C.byref(desc.c), int(hoist), buf, need.value, C.byref(need)))
    return buf.value.decode()


def jit_compile(scene: dict[str, Any] | SceneDesc, hoist: bool = True) -> tuple[int, str]:
    """NVRTC-compile a scene's material module for sm_100a (no GPU needed): (cubin bytes, log)."""
    desc = scene if isinstance(scene, SceneDesc) else SceneDesc(scene)
    log = C.create_string_buffer(1 << 16)
    nbytes = C.c_int64()
    check(lib().rmd_test_jit_compile(C.byref(desc.c), int(hoist), log, 1 << 16, C.byref(nbytes)))
    return nbytes.value, log.value.decode(errors="replace")


def _exr_compression(name: str) -> int:
    table = {"auto": _abi.EXR_AUTO, "none": _abi.EXR_NONE, "zip": _abi.EXR_ZIP}
    if name not in table:
        raise ValueError(f"compression must be one of {sorted(table)}, not {name!r}")
    return table[name]


def test_exr_write(path, rgb: np.ndarray, normalized_by: float = 1.0, compression: str = "auto") -> None:
    """Test hook: the film EXR writer applied to a host image (h, w, 3)."""
    a = np.ascontiguousarray(rgb, np.float32)
    check(lib().rmd_test_exr_write(str(path).encode(), _f32p(a), a.shape[1], a.shape[0], normalized_by,
                                   _exr_compression(compression)))


def test_prng(mode: int, a: int, b: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    check(lib().rmd_test_prng(mode, a, b, n, _f32p(out)))
    return out
