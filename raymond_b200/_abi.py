"""ctypes mirror of include/raymond.h.

The structs below are field-for-field the C declarations; `SceneDesc` builds
an `rmd_scene_desc` from numpy arrays and node-graph dictionaries and keeps
every buffer alive for as long as the descriptor object lives.
"""
from __future__ import annotations

import ctypes as C
from typing import Any

import numpy as np

RMD_OK = 0
STATUS_NAMES = {
    0: "RMD_OK", 1: "RMD_ERROR_INVALID_ARGUMENT", 2: "RMD_ERROR_CUDA", 3: "RMD_ERROR_NVRTC",
    4: "RMD_ERROR_CODEGEN_CYCLE", 5: "RMD_ERROR_CODEGEN_MULTI_INPUT", 6: "RMD_ERROR_CODEGEN_UNSUPPORTED",
    7: "RMD_ERROR_OUT_OF_MEMORY", 8: "RMD_ERROR_QUEUE_OVERFLOW", 9: "RMD_ERROR_WATCHDOG",
    10: "RMD_ERROR_NO_DEVICE",
}

RAY_CAMERA, RAY_REFLECTION, RAY_TRANSMISSION, RAY_SHADOW = 1, 2, 4, 8
RAY_VOLUME, RAY_DIFFUSE, RAY_GLOSSY, RAY_SINGULAR = 16, 32, 64, 128
VISIBLE_ALL = RAY_CAMERA | RAY_DIFFUSE | RAY_GLOSSY | RAY_TRANSMISSION | RAY_VOLUME | RAY_SHADOW

SAMPLING_BSDF, SAMPLING_NEE, SAMPLING_MIS = 0, 1, 2
TONEMAP_LINEAR, TONEMAP_HABLE, TONEMAP_ACES = 0, 1, 2
RNG_PCG32, RNG_TEA = 0, 1

PARAM_STRING, PARAM_NUMBER, PARAM_BOOL, PARAM_NUMBERS = 0, 1, 2, 3


def _layout(fields):
    """ctypes fields laid out as C lays out the header's structs, including
    members declared RMD_ALIGN(n): entries are (name, type) or (name, type,
    alignment).  Padding fields (_padN) are inserted where C pads, so nested
    records and arrays of them have the C offsets and sizes.  Returns the
    fields and the struct's alignment."""
    out, off, align, npad = [], 0, 1, 0
    for f in fields:
        name, typ = f[0], f[1]
        a = max(f[2] if len(f) > 2 else 1, getattr(typ, "_rmd_align_", C.alignment(typ)))
        if off % a:
            out.append((f"_pad{npad}", C.c_uint8 * (a - off % a)))
            npad += 1
            off += a - off % a
        out.append((name, typ))
        off += C.sizeof(typ)
        align = max(align, a)
    if off % align:
        out.append((f"_pad{npad}", C.c_uint8 * (align - off % align)))
    return out, align


class NodeParam(C.Structure):
    _fields_ = [("key", C.c_char_p), ("kind", C.c_int32), ("string_value", C.c_char_p),
                ("number_value", C.c_double), ("numbers", C.POINTER(C.c_float)), ("num_numbers", C.c_int32)]


class NodeInput(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_char_p), ("num_values", C.c_int32),
                ("values", C.c_float * 4), ("link_node", C.c_char_p), ("link_socket", C.c_char_p),
                ("num_links", C.c_int32)]


class Node(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_char_p), ("num_inputs", C.c_int32),
                ("inputs", C.POINTER(NodeInput)), ("num_params", C.c_int32), ("params", C.POINTER(NodeParam))]


class Material(C.Structure):
    _fields_ = [("name", C.c_char_p), ("num_nodes", C.c_int32), ("nodes", C.POINTER(Node))]


class Shape(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_faces", C.c_uint32),
                ("vertices", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("texcoords", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_uint32)),
                ("materials", C.POINTER(C.c_uint16))]


class Entity(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("visibility", C.c_uint32), ("matrix", C.c_float * 16)]


class LightInfo(C.Structure):
    _fields_ = [("shader_index", C.c_uint16), ("casts_shadows", C.c_uint8), ("uses_mis", C.c_uint8)]


class AreaLight(C.Structure):  # bridge/lights/AreaLight.hpp, 96 bytes
    _fields_, _rmd_align_ = _layout([("info", LightInfo), ("transform", C.c_float * 12, 16),
                                     ("color", C.c_float * 4, 16), ("is_circular", C.c_uint8)])


class PointLight(C.Structure):  # bridge/lights/PointLight.hpp, 64 bytes
    _fields_, _rmd_align_ = _layout([("info", LightInfo), ("location", C.c_float * 4, 16), ("radius", C.c_float),
                                     ("color", C.c_float * 4, 16)])


class SunLight(C.Structure):  # bridge/lights/SunLight.hpp, 64 bytes
    _fields_, _rmd_align_ = _layout([("info", LightInfo), ("direction", C.c_float * 4, 16),
                                     ("cos_angle", C.c_float), ("color", C.c_float * 4, 16)])


class SpotLight(C.Structure):  # bridge/lights/SpotLight.hpp, 96 bytes
    _fields_, _rmd_align_ = _layout([("info", LightInfo), ("location", C.c_float * 4, 16),
                                     ("direction", C.c_float * 4, 16), ("radius", C.c_float),
                                     ("color", C.c_float * 4, 16), ("spot_size", C.c_float),
                                     ("spot_blend", C.c_float)])


class Camera(C.Structure):  # bridge/Camera.hpp, 96 bytes
    _fields_, _rmd_align_ = _layout([("transform", C.c_float * 16, 16), ("near_clip", C.c_float),
                                     ("far_clip", C.c_float), ("focal_length", C.c_float),
                                     ("shift", C.c_float * 2, 8)])


class PerInstanceData(C.Structure):  # bridge/PerInstanceData.hpp, 192 bytes
    _fields_, _rmd_align_ = _layout([("vertex_offset", C.c_uint32), ("face_offset", C.c_uint32),
                                     ("light_face_offset", C.c_uint32), ("light_face_count", C.c_uint32),
                                     ("light_index", C.c_uint32), ("bounds_min", C.c_float * 4, 16),
                                     ("bounds_size", C.c_float * 4, 16), ("point_transform", C.c_float * 16, 16),
                                     ("normal_transform", C.c_float * 12, 16), ("visibility", C.c_uint8)])


OUTPUT_IMAGE, RR_NONE, RR_THROUGHPUT = 0, 0, 1


class Uniforms(C.Structure):  # bridge/Uniforms.hpp, 64 bytes
    _fields_, _rmd_align_ = _layout([("num_lens_surfaces", C.c_uint32), ("frame_index", C.c_uint32),
                                     ("random_seed", C.c_uint32), ("accumulate", C.c_uint8),
                                     ("lens_spectral", C.c_uint8), ("sensor_scale", C.c_float),
                                     ("camera_scale", C.c_float), ("focus", C.c_float), ("exposure", C.c_float),
                                     ("stop_index", C.c_int32), ("relative_stop", C.c_float),
                                     ("num_aperture_blades", C.c_int32), ("sampling_mode", C.c_uint32),
                                     ("tonemapping", C.c_uint32), ("rr", C.c_uint32), ("rr_depth", C.c_int32),
                                     ("output_channel", C.c_uint32)])


def default_uniforms(**kw) -> Uniforms:
    """The reference's initial Uniforms (Renderer.swift:331-349), with `kw` overrides."""
    u = Uniforms(num_lens_surfaces=0, frame_index=0, random_seed=1, accumulate=1, lens_spectral=1,
                 sensor_scale=1.0, camera_scale=0.001, focus=0.0, exposure=1.0, stop_index=0, relative_stop=1.0,
                 num_aperture_blades=7, sampling_mode=SAMPLING_MIS, tonemapping=TONEMAP_LINEAR, rr=RR_THROUGHPUT,
                 rr_depth=0, output_channel=OUTPUT_IMAGE)
    for k, v in kw.items():
        setattr(u, k, v)
    return u


class BatchView(C.Structure):
    _fields_, _rmd_align_ = _layout([("scene", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32),
                                     ("camera", Camera)])


BATCH_NO_GRAPH = 1


TEXTURE_U8, TEXTURE_U16, TEXTURE_F32 = 0, 1, 2


class Texture(C.Structure):
    _fields_ = [("name", C.c_char_p), ("width", C.c_uint32), ("height", C.c_uint32), ("channels", C.c_uint32),
                ("format", C.c_uint32), ("data", C.c_void_p)]


class SceneDescC(C.Structure):
    _fields_, _rmd_align_ = _layout([
        ("num_surface_materials", C.c_int32), ("surface_materials", C.POINTER(Material)),
        ("num_light_materials", C.c_int32), ("light_materials", C.POINTER(Material)),
        ("num_shapes", C.c_int32), ("shapes", C.POINTER(Shape)),
        ("num_entities", C.c_int32), ("entities", C.POINTER(Entity)),
        ("world_shader", C.c_uint16), ("envmap_exponent", C.c_int32),
        ("num_area_lights", C.c_int32), ("area_lights", C.POINTER(AreaLight)),
        ("num_point_lights", C.c_int32), ("point_lights", C.POINTER(PointLight)),
        ("num_sun_lights", C.c_int32), ("sun_lights", C.POINTER(SunLight)),
        ("num_spot_lights", C.c_int32), ("spot_lights", C.POINTER(SpotLight)),
        ("camera", Camera), ("num_textures", C.c_int32), ("textures", C.POINTER(Texture))])


class RenderSettings(C.Structure):
    _fields_ = [("spp", C.c_uint32), ("max_depth", C.c_uint32), ("sampling_mode", C.c_uint32),
                ("rng", C.c_uint32), ("seed", C.c_uint64), ("first_sample", C.c_int64),
                ("film_fp64", C.c_uint32), ("reserved", C.c_uint32)]


class TuneResult(C.Structure):
    _fields_ = [("shade_min_blocks", C.c_uint32), ("trace_blocks_per_sm", C.c_uint32), ("pool_size", C.c_uint32),
                ("calibration_spp", C.c_uint32), ("ms_default", C.c_double), ("ms_best", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("segments", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("iterations", C.c_uint64), ("ms_total", C.c_double), ("ms_trace", C.c_double),
                ("ms_shade", C.c_double), ("ms_shadow", C.c_double), ("ms_film", C.c_double),
                ("pool_size", C.c_uint32), ("errors", C.c_uint32), ("rays", C.c_uint64),
                ("ms_guide", C.c_double), ("ms_guide_train", C.c_double), ("invalid_samples", C.c_uint64)]


class GuideSettings(C.Structure):
    _fields_ = [("sampling", C.c_uint32), ("training", C.c_uint32), ("batch_size", C.c_uint32),
                ("learning_rate", C.c_float), ("reset", C.c_uint32), ("seed", C.c_uint32),
                ("step_records", C.c_uint32), ("replay_records", C.c_uint32), ("steps_per_batch", C.c_uint32),
                ("skip_light_records", C.c_uint32), ("guided_depth", C.c_uint32)]


class GuideStats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("samples", C.c_uint64), ("records", C.c_uint64), ("last_loss", C.c_float),
                ("reserved", C.c_float)]


EXR_AUTO = 0
EXR_NONE = 1
EXR_ZIP = 2
BVH_HOST = 0
BVH_GPU = 1
BVH_BUILDERS = {"host": BVH_HOST, "gpu": BVH_GPU}


class BvhStats(C.Structure):
    _fields_ = [("builder", C.c_uint32), ("levels", C.c_uint32), ("nodes", C.c_uint64), ("build_ms", C.c_double),
                ("sah_cost", C.c_double), ("cluster_iterations", C.c_uint32), ("reserved", C.c_uint32)]


def _fptr(a: np.ndarray, ctype=C.c_float):
    return a.ctypes.data_as(C.POINTER(ctype))


class SceneDesc:
    """Owns the C descriptor of one scene plus every array it points to.

    `scene` is the dictionary produced by `raymond_b200.scenes` (or by a user):
      materials:       list of (name, node-graph dict in the exporter's format)
      light_materials: list of (name, node-graph dict)
      shapes:          list of dicts with vertices (V,3) f32, normals (V,3),
                       texcoords (V,2), indices (F,3) u32, materials (F,) u16
      entities:        list of dicts {shape, matrix (4,4) row-major world matrix, visibility}
      world_shader, envmap_exponent, area/point/sun/spot light lists, camera dict
      textures:        optional {file path: (height, width[, 1|3|4]) uint8, uint16 or
                       float32 image, top row first} for image / environment texture nodes
    """

    def __init__(self, scene: dict[str, Any]):
        self._keep: list[Any] = []
        self.scene = scene
        d = SceneDescC()
        surf = [self._material(n, g) for n, g in scene["materials"]]
        lmat = [self._material(n, g) for n, g in scene["light_materials"]]
        d.num_surface_materials = len(surf)
        d.surface_materials = self._array(Material, surf)
        d.num_light_materials = len(lmat)
        d.light_materials = self._array(Material, lmat)

        shapes = []
        for s in scene["shapes"]:
            v = np.ascontiguousarray(s["vertices"], dtype=np.float32)
            n = np.ascontiguousarray(s["normals"], dtype=np.float32)
            t = np.ascontiguousarray(s["texcoords"], dtype=np.float32)
            i = np.ascontiguousarray(s["indices"], dtype=np.uint32)
            m = np.ascontiguousarray(s["materials"], dtype=np.uint16)
            self._keep += [v, n, t, i, m]
            shapes.append(Shape(len(v), len(i), _fptr(v), _fptr(n), _fptr(t), _fptr(i, C.c_uint32),
                                _fptr(m, C.c_uint16)))
        d.num_shapes = len(shapes)
        d.shapes = self._array(Shape, shapes)

        ents = []
        for e in scene["entities"]:
            mat = np.asarray(e["matrix"], dtype=np.float32).reshape(4, 4)
            ent = Entity()
            ent.shape = e["shape"]
            ent.visibility = e.get("visibility", VISIBLE_ALL)
            ent.matrix[:] = mat.T.reshape(-1).tolist()  # column-major
            ents.append(ent)
        d.num_entities = len(ents)
        d.entities = self._array(Entity, ents)

        d.world_shader = scene.get("world_shader", 0)
        d.envmap_exponent = scene.get("envmap_exponent", 11)

        def info(l):
            return LightInfo(l.get("shader", 0), int(l.get("casts_shadows", True)), 0)

        areas = []
        for l in scene.get("area_lights", []):
            a = AreaLight()
            a.info = info(l)
            a.transform[:] = np.asarray(l["transform"], np.float32).reshape(3, 4).reshape(-1).tolist()
            a.color[:3] = list(l["color"])
            a.is_circular = int(l.get("is_circular", False))
            areas.append(a)
        points = []
        for l in scene.get("point_lights", []):
            p = PointLight()
            p.info = info(l)
            p.location[:3] = list(l["location"])
            p.radius = l.get("radius", 0.0)
            p.color[:3] = list(l["color"])
            points.append(p)
        suns = []
        for l in scene.get("sun_lights", []):
            s = SunLight()
            s.info = info(l)
            dvec = np.asarray(l["direction"], np.float64)
            s.direction[:3] = (dvec / np.linalg.norm(dvec)).tolist()
            s.cos_angle = float(np.cos(l.get("angle", 0.0) / 2))
            s.color[:3] = list(l["color"])
            suns.append(s)
        spots = []
        for l in scene.get("spot_lights", []):
            s = SpotLight()
            s.info = info(l)
            s.location[:3] = list(l["location"])
            dvec = np.asarray(l["direction"], np.float64)
            s.direction[:3] = (dvec / np.linalg.norm(dvec)).tolist()
            s.radius = l.get("radius", 0.0)
            s.color[:3] = list(l["color"])
            ang = float(np.cos(l["spot_size"] / 2))
            s.spot_size = ang
            s.spot_blend = (1 - ang) * l.get("spot_blend", 0.0)
            spots.append(s)
        d.num_area_lights, d.area_lights = len(areas), self._array(AreaLight, areas)
        d.num_point_lights, d.point_lights = len(points), self._array(PointLight, points)
        d.num_sun_lights, d.sun_lights = len(suns), self._array(SunLight, suns)
        d.num_spot_lights, d.spot_lights = len(spots), self._array(SpotLight, spots)
        d.camera = make_camera(scene["camera"])
        texs = []
        for name, img in scene.get("textures", {}).items():
            a = np.ascontiguousarray(img)
            if a.ndim == 2:
                a = a[:, :, None]
            if a.ndim != 3 or a.shape[2] not in (1, 3, 4):
                raise ValueError(f"texture {name!r}: expected (height, width, 1|3|4), got {a.shape}")
            fmt = {np.dtype(np.uint8): TEXTURE_U8, np.dtype(np.uint16): TEXTURE_U16}.get(a.dtype, TEXTURE_F32)
            if fmt == TEXTURE_F32:
                a = np.ascontiguousarray(a, np.float32)
            self._keep.append(a)
            texs.append(Texture(self._str(name), a.shape[1], a.shape[0], a.shape[2], fmt, a.ctypes.data))
        d.num_textures, d.textures = len(texs), self._array(Texture, texs)
        self.c = d

    def _array(self, T, items):
        arr = (T * max(1, len(items)))(*items)
        self._keep.append(arr)
        return C.cast(arr, C.POINTER(T))

    def _str(self, s: str):
        b = C.c_char_p(s.encode())
        self._keep.append(b)
        return b.value

    def _material(self, name: str, graph: dict[str, Any]) -> Material:
        nodes = []
        for node_name, node in graph.items():
            inputs = []
            for in_name, inp in node.get("inputs", {}).items():
                ni = NodeInput()
                ni.name = self._str(in_name)
                ni.type = self._str(inp.get("type", "VALUE"))
                links = inp.get("links") or []
                ni.num_links = len(links)
                if links:
                    ni.link_node = self._str(links[0][0])
                    ni.link_socket = self._str(links[0][1])
                val = inp.get("value")
                if val is not None and not isinstance(val, str):
                    if isinstance(val, (list, tuple)):
                        ni.num_values = len(val)
                        for k, x in enumerate(val[:4]):
                            ni.values[k] = float(x)
                    else:
                        ni.num_values = 1
                        ni.values[0] = float(val)
                inputs.append(ni)
            params = []
            for key, val in node.get("parameters", {}).items():
                p = NodeParam()
                p.key = self._str(key)
                if isinstance(val, bool):
                    p.kind, p.number_value = PARAM_BOOL, float(val)
                elif isinstance(val, (int, float)):
                    p.kind, p.number_value = PARAM_NUMBER, float(val)
                elif isinstance(val, str):
                    p.kind, p.string_value = PARAM_STRING, self._str(val)
                elif isinstance(val, (list, tuple)):
                    flat: list[float] = []
                    for x in val:
                        if isinstance(x, dict):  # ColorRamp element
                            flat.append(float(x["position"]))
                            flat.extend(float(c) for c in x["color"])
                        else:
                            flat.append(float(x))
                    arr = np.asarray(flat, dtype=np.float32)
                    self._keep.append(arr)
                    p.kind, p.numbers, p.num_numbers = PARAM_NUMBERS, _fptr(arr), len(flat)
                else:
                    continue
                params.append(p)
            n = Node()
            n.name = self._str(node_name)
            n.type = self._str(node["type"])
            n.num_inputs, n.inputs = len(inputs), self._array(NodeInput, inputs)
            n.num_params, n.params = len(params), self._array(NodeParam, params)
            nodes.append(n)
        m = Material()
        m.name = self._str(name)
        m.num_nodes, m.nodes = len(nodes), self._array(Node, nodes)
        return m


def make_camera(cam: dict[str, Any]) -> Camera:
    c = Camera()
    mat = np.asarray(cam["transform"], dtype=np.float32).reshape(4, 4)
    c.transform[:] = mat.T.reshape(-1).tolist()  # column-major
    c.near_clip = cam.get("near_clip", 0.1)
    c.far_clip = cam.get("far_clip", 100.0)
    c.focal_length = cam.get("focal_length", 2.5)
    sh = cam.get("shift", (0.0, 0.0))
    c.shift[0], c.shift[1] = sh[0], sh[1]
    return c
