"""Scene files in the reference's on-disk format: the JSON its Blender exporter
writes (scripts/blender_exporter/raymond_blender/exporter.py:49-69) and the
ASCII PLY meshes beside it (shapes.py:20-129), read the way the reference's
host reads them.

`load_scene(path)` returns the scene dictionary `raymond_b200.SceneDesc`
takes, plus the render resolution of the file.  `save_scene` writes a scene
dictionary in the same format (meshes under `meshes/`), so scenes built here
round-trip through the reference's format.

Reading rules kept from the reference:

* PLY numbers are parsed as the reference's `my_strtof` does
  (io/PLYReader.m:63-97): the digits form an integer, the value is that
  integer (as a float) times powf(10, -digits after the point), not the
  correctly rounded decimal.  Faces are triangles "3 i j k m" whose last
  entry indexes the shape's material list (PLYReader.m:143-167).
* Camera focal length = lens / (sensor width / 2), 50 mm when absent
  (SceneLoader.swift:135-136).
* Light records as LightBuilder.build makes them (LightBuilder.swift:187-220):
  colour x power (x 4/pi for circular area lights), spot size as the cosine
  of its half angle and blend scaled by (1 - that cosine), sun angle as the
  cosine of its half angle, directions normalised.
* Visibility flags from the exporter's booleans (EntityBuilder.swift:55-64).
* Image and environment texture nodes name their image file (relative to the
  scene file); PNG and OpenEXR files, the formats the exporter writes
  (materials.py:194-209), are read into `scene["textures"]`.  A file that is
  absent or in another format is left out with a warning, and the node then
  reads the 1 x 1 zero texture, as the reference does when MTKTextureLoader
  fails (MaterialBuilder.swift:224-234).
"""
from __future__ import annotations

import json
import os
import warnings
from pathlib import Path
from typing import Any

import numpy as np

from ._abi import RAY_CAMERA, RAY_DIFFUSE, RAY_GLOSSY, RAY_SHADOW, RAY_TRANSMISSION, RAY_VOLUME, VISIBLE_ALL

_VISIBILITY = {"camera": RAY_CAMERA, "diffuse": RAY_DIFFUSE, "glossy": RAY_GLOSSY,
               "transmission": RAY_TRANSMISSION, "volume": RAY_VOLUME, "shadow": RAY_SHADOW}


class SceneFormatError(ValueError):
    pass


# ---------------------------------------------------------------------- PLY
def parse_reference_floats(tokens: np.ndarray) -> np.ndarray:
    """Decimal strings -> float32 the way the reference's PLY reader parses
    them: integer of all digits times powf(10, -(digits after the point))."""
    toks = np.asarray(tokens, dtype=str)
    neg = np.char.startswith(toks, "-")
    body = np.where(neg, np.char.lstrip(toks, "-"), toks)
    parts = np.char.partition(body, ".")
    frac_digits = np.char.str_len(parts[..., 2])
    digits = np.char.add(parts[..., 0], parts[..., 2])
    ok = np.char.isdigit(digits)
    if not ok.all():
        bad = toks[~ok][0]
        raise SceneFormatError(f"PLY number {bad!r} is not a plain decimal")
    decimal = digits.astype(np.int64)
    decimal = np.where(neg, -decimal, decimal)
    # powf(10, e) for the small exponents the exporter writes, correctly rounded
    scale = np.array([np.float32(10.0 ** (-k)) for k in range(0, 19)], np.float32)
    if frac_digits.max(initial=0) > 18:
        raise SceneFormatError("PLY number with more than 18 decimals")
    return (decimal.astype(np.float32) * scale[frac_digits]).astype(np.float32)


def read_ply(path: str | os.PathLike) -> dict[str, np.ndarray]:
    """ASCII PLY of the exporter: x y z nx ny nz s t per vertex; faces of 3
    indices and a material-palette index."""
    with open(path, "rb") as f:
        raw = f.read()
    head_end = raw.find(b"end_header\n")
    if not raw.startswith(b"ply\n") or head_end < 0:
        raise SceneFormatError(f"{path}: not a PLY file")
    header = raw[:head_end].decode().splitlines()
    if "format ascii 1.0" not in header:
        raise SceneFormatError(f"{path}: only ASCII PLY is supported")
    counts = {}
    for line in header:
        p = line.split()
        if p and p[0] == "element":
            counts[p[1]] = int(p[2])
    nv, nf = counts.get("vertex", 0), counts.get("face", 0)
    lines = raw[head_end + len(b"end_header\n"):].decode().split("\n")
    if len(lines) < nv + nf:
        raise SceneFormatError(f"{path}: {len(lines)} data lines for {nv} vertices and {nf} faces")
    vtok = np.array([ln.split() for ln in lines[:nv]], dtype=str).reshape(nv, 8) if nv else np.zeros((0, 8), str)
    vals = parse_reference_floats(vtok.reshape(-1)).reshape(nv, 8) if nv else np.zeros((0, 8), np.float32)
    ftok = [ln.split() for ln in lines[nv:nv + nf]]
    if any(len(t) != 5 or t[0] != "3" for t in ftok):
        raise SceneFormatError(f"{path}: faces must be triangles with a material index")
    faces = np.array(ftok, dtype=np.int64).reshape(nf, 5) if nf else np.zeros((0, 5), np.int64)
    if nf and (faces[:, 1:4].max() >= nv or faces[:, 1:4].min() < 0):
        raise SceneFormatError(f"{path}: face index out of range")
    return {"vertices": vals[:, 0:3].copy(), "normals": vals[:, 3:6].copy(), "texcoords": vals[:, 6:8].copy(),
            "indices": faces[:, 1:4].astype(np.uint32), "palette": faces[:, 4].astype(np.int64)}


def write_ply(path: str | os.PathLike, shape: dict[str, np.ndarray], palette: np.ndarray) -> None:
    """The exporter's ASCII PLY (shapes.py:20-129): %.6f numbers."""
    v, n, t = (np.asarray(shape[k], np.float64) for k in ("vertices", "normals", "texcoords"))
    idx = np.asarray(shape["indices"], np.int64)
    rows = [f"{a:.6f} {b:.6f} {c:.6f} {d:.6f} {e:.6f} {f_:.6f} {g:.6f} {h:.6f}"
            for (a, b, c), (d, e, f_), (g, h) in zip(v, n, t)]
    frows = [f"3 {i} {j} {k} {m}" for (i, j, k), m in zip(idx, palette)]
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\ncomment Copyright raymond exporter research team\n")
        f.write(f"element vertex {len(v)}\nproperty float x\nproperty float y\nproperty float z\n"
                "property float nx\nproperty float ny\nproperty float nz\nproperty float s\nproperty float t\n")
        f.write(f"element face {len(idx)}\nproperty list uchar uint vertex_indices\nproperty uchar material_index\n"
                "end_header\n")
        f.write("\n".join(rows + frows) + "\n")


# ---------------------------------------------------------------------- JSON
def _visibility(v: dict[str, bool] | None) -> int:
    if v is None:
        return sum(_VISIBILITY.values())
    return sum(bit for key, bit in _VISIBILITY.items() if v.get(key, True))


def load_scene(path: str | os.PathLike) -> tuple[dict[str, Any], tuple[int, int] | None]:
    """Scene dictionary and render resolution of an exporter JSON file."""
    path = Path(path)
    doc = json.loads(path.read_text())
    materials: dict[str, Any] = doc.get("materials", {})
    lights: dict[str, Any] = doc.get("lights", {})
    # materials used by lights form the light table; those used by shapes, and
    # any used by nothing, the surface table (a material may be in both)
    light_names: list[str] = []
    for light in lights.values():
        if light["material"] not in light_names:
            light_names.append(light["material"])
    shape_refs = {m for sd in doc.get("shapes", {}).values() for m in sd.get("materials", [])}
    surface_names = [n for n in materials if n in shape_refs or n not in light_names]
    for n in light_names:
        if n not in materials:
            raise SceneFormatError(f"light material {n!r} is not defined")
    surface_index = {n: i for i, n in enumerate(surface_names)}
    light_index = {n: i for i, n in enumerate(light_names)}

    shapes, shape_index = [], {}
    for name, sd in doc.get("shapes", {}).items():
        if sd.get("type", "ply") != "ply":
            raise SceneFormatError(f"shape {name!r}: unsupported type {sd.get('type')!r}")
        mesh = read_ply(path.parent / sd["filepath"])
        names = sd.get("materials", [])
        pal = []
        for m in names:
            if m not in surface_index:
                raise SceneFormatError(f"shape {name!r}: material {m!r} is not a surface material")
            pal.append(surface_index[m])
        if len(mesh["palette"]) and mesh["palette"].max() >= len(pal):
            raise SceneFormatError(f"shape {name!r}: face material index beyond its {len(pal)} materials")
        mats = np.asarray(pal, np.uint16)[mesh["palette"]] if len(pal) else np.zeros(len(mesh["indices"]), np.uint16)
        shape_index[name] = len(shapes)
        shapes.append({"vertices": mesh["vertices"], "normals": mesh["normals"], "texcoords": mesh["texcoords"],
                       "indices": mesh["indices"], "materials": mats})

    entities = []
    for name, ed in doc.get("entities", {}).items():
        if ed["shape"] not in shape_index:
            raise SceneFormatError(f"entity {name!r}: unknown shape {ed['shape']!r}")
        entities.append({"shape": shape_index[ed["shape"]],
                         "matrix": np.asarray(ed["matrix"], np.float32).reshape(4, 4),
                         "visibility": _visibility(ed.get("visibility"))})

    scene: dict[str, Any] = {
        "materials": [(n, materials[n]) for n in surface_names],
        "light_materials": [(n, materials[n]) for n in light_names],
        "shapes": shapes, "entities": entities,
        "area_lights": [], "point_lights": [], "sun_lights": [], "spot_lights": [],
        "envmap_exponent": 11,  # LightBuilder.swift:97
    }
    world = None
    for name, ld in lights.items():
        kind, p = ld["type"], ld.get("parameters", {})
        base = {"shader": light_index[ld["material"]], "casts_shadows": bool(ld.get("cast_shadows", True))}
        color = np.asarray(p.get("color", [1, 1, 1]), np.float64)[:3] * float(p.get("power", 1.0))
        if kind == "WORLD":
            world = light_index[ld["material"]]
        elif kind == "AREA":
            norm = 4.0 / np.pi if p.get("is_circular", False) else 1.0
            scene["area_lights"].append({**base, "transform": np.asarray(p["transform"], np.float32).reshape(4, 4)[:3],
                                         "color": tuple(norm * color), "is_circular": bool(p.get("is_circular", False))})
        elif kind == "POINT":
            scene["point_lights"].append({**base, "location": tuple(p["location"]), "radius": float(p.get("radius", 0)),
                                          "color": tuple(color)})
        elif kind == "SUN":
            scene["sun_lights"].append({**base, "direction": tuple(p["direction"]), "angle": float(p.get("angle", 0)),
                                        "color": tuple(color)})
        elif kind == "SPOT":
            scene["spot_lights"].append({**base, "location": tuple(p["location"]), "direction": tuple(p["direction"]),
                                         "radius": float(p.get("radius", 0)), "color": tuple(color),
                                         "spot_size": float(p["spot_size"]), "spot_blend": float(p.get("spot_blend", 0))})
        else:
            raise SceneFormatError(f"light {name!r}: unsupported type {kind!r}")
    if world is None:
        raise SceneFormatError("the scene has no WORLD light")
    scene["world_shader"] = world

    cam = doc.get("camera")
    if cam:
        film_w = float(cam.get("film", {}).get("width", 36.0))
        scene["camera"] = {"transform": np.asarray(cam["transform"], np.float32).reshape(4, 4),
                           "near_clip": float(cam.get("near_clip", 0.1)), "far_clip": float(cam.get("far_clip", 100.0)),
                           "focal_length": float(cam.get("focal_length", 50.0)) / (film_w / 2),
                           "shift": tuple(cam.get("shift", (0.0, 0.0)))}
    else:  # SceneLoader.makeDefaultCamera (SceneLoader.swift:30-41)
        scene["camera"] = {"transform": np.eye(4, dtype=np.float32), "near_clip": 0.1, "far_clip": 100.0,
                           "focal_length": 2.5, "shift": (0.0, 0.0)}
    scene["textures"] = _read_textures(path.parent, list(materials.values()))
    res = doc.get("render", {}).get("resolution")
    size = (int(res["width"]), int(res["height"])) if res else None
    return scene, size


def read_image(path: str | os.PathLike) -> np.ndarray:
    """A PNG (uint8 / uint16) or OpenEXR (float32) image as (height, width, channels)."""
    from . import exr, png

    p = Path(path)
    head = p.read_bytes()[:8]
    if head.startswith(b"\x89PNG"):
        return png.read_png(p)
    if head[:4] == bytes([0x76, 0x2F, 0x31, 0x01]):
        ch, _ = exr.read_exr(p)
        if set("RGB") <= set(ch):
            names = ["R", "G", "B"] + (["A"] if "A" in ch else [])
        elif "Y" in ch:
            names = ["Y"]
        else:
            names = sorted(ch)[:4]
        return np.stack([ch[n] for n in names], axis=-1).astype(np.float32)
    raise SceneFormatError(f"{p.name}: not a PNG or OpenEXR image")


def _read_textures(base: Path, graphs: list) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    for graph in graphs:
        for node in graph.values():
            if node.get("type") not in ("TEX_IMAGE", "TEX_ENVIRONMENT"):
                continue
            file = node.get("parameters", {}).get("filepath")
            if not file or file in out:
                continue
            try:
                out[file] = read_image(base / file)
            except (OSError, ValueError) as e:
                warnings.warn(f"texture {file!r} not loaded ({e}); the node reads a 1 x 1 zero texture")
    return out


def save_scene(scene: dict[str, Any], path: str | os.PathLike, resolution: tuple[int, int] | None = None) -> None:
    """Writes a scene dictionary in the exporter's format (JSON + meshes/*.ply).
    Lights are written with power 1 and their colour as it is in the
    dictionary (the reader multiplies by the power)."""
    path = Path(path)
    (path.parent / "meshes").mkdir(parents=True, exist_ok=True)
    mats = {n: g for n, g in scene["materials"]}
    lmats = {n: g for n, g in scene["light_materials"]}
    clash = set(mats) & set(lmats)
    if clash:
        raise SceneFormatError(f"material names used for both surfaces and lights: {sorted(clash)}")
    snames = [n for n, _ in scene["materials"]]
    lnames = [n for n, _ in scene["light_materials"]]
    shapes = {}
    for i, s in enumerate(scene["shapes"]):
        used = sorted(set(int(m) for m in np.asarray(s["materials"]).tolist()))
        pal = {m: k for k, m in enumerate(used)}
        write_ply(path.parent / "meshes" / f"shape{i}.ply", s, np.array([pal[int(m)] for m in s["materials"]]))
        shapes[f"shape{i}"] = {"type": "ply", "filepath": f"meshes/shape{i}.ply", "materials": [snames[m] for m in used]}
    vis_of = lambda bits: {k: bool(bits & b) for k, b in _VISIBILITY.items()}
    entities = {f"entity{i}": {"shape": f"shape{e['shape']}", "visibility": vis_of(e.get("visibility", VISIBLE_ALL)),
                               "matrix": np.asarray(e["matrix"], np.float64).reshape(-1).tolist()}
                for i, e in enumerate(scene["entities"])}
    lights = {"world": {"type": "WORLD", "material": lnames[scene.get("world_shader", 0)], "cast_shadows": True,
                        "use_mis": True}}

    def entry(kind, l, params):
        return {"type": kind, "material": lnames[l.get("shader", 0)], "cast_shadows": bool(l.get("casts_shadows", True)),
                "use_mis": False, "parameters": {**params, "power": 1.0}}
    for i, l in enumerate(scene.get("area_lights", [])):
        circ = bool(l.get("is_circular", False))
        t = np.vstack([np.asarray(l["transform"], np.float64).reshape(3, 4), [0, 0, 0, 1]])
        col = np.asarray(l["color"], np.float64) / (4.0 / np.pi if circ else 1.0)
        lights[f"area{i}"] = entry("AREA", l, {"transform": t.reshape(-1).tolist(), "color": col.tolist(),
                                                "spread": np.pi, "is_circular": circ})
    for i, l in enumerate(scene.get("point_lights", [])):
        lights[f"point{i}"] = entry("POINT", l, {"location": list(l["location"]), "color": list(l["color"]),
                                                  "radius": l.get("radius", 0.0)})
    for i, l in enumerate(scene.get("sun_lights", [])):
        lights[f"sun{i}"] = entry("SUN", l, {"direction": list(l["direction"]), "color": list(l["color"]),
                                              "angle": l.get("angle", 0.0)})
    for i, l in enumerate(scene.get("spot_lights", [])):
        lights[f"spot{i}"] = entry("SPOT", l, {"location": list(l["location"]), "direction": list(l["direction"]),
                                                "color": list(l["color"]), "radius": l.get("radius", 0.0),
                                                "spot_size": l["spot_size"], "spot_blend": l.get("spot_blend", 0.0)})
    cam = scene["camera"]
    doc = {"materials": {**mats, **lmats}, "shapes": shapes, "entities": entities, "lights": lights,
           "camera": {"near_clip": cam.get("near_clip", 0.1), "far_clip": cam.get("far_clip", 100.0),
                      "film": {"width": 36.0, "height": 24.0},
                      "transform": np.asarray(cam["transform"], np.float64).reshape(-1).tolist(),
                      "shift": list(cam.get("shift", (0.0, 0.0))), "type": "perspective",
                      "focal_length": cam.get("focal_length", 2.5) * 18.0}}
    if resolution:
        doc["render"] = {"resolution": {"width": resolution[0], "height": resolution[1]}}
    from . import exr, png

    for name, img in scene.get("textures", {}).items():  # beside the scene file, where the nodes name them
        out = path.parent / name
        out.parent.mkdir(parents=True, exist_ok=True)
        a = np.asarray(img)
        if a.dtype in (np.uint8, np.uint16) and out.suffix.lower() == ".png":
            png.write_png(out, a, filters=(0, 1, 2, 3, 4))
        elif out.suffix.lower() == ".exr":
            exr.write_exr(out, a)
        else:
            raise SceneFormatError(f"texture {name!r}: PNG needs uint8 / uint16 data, other images an .exr name")
    path.write_text(json.dumps(doc, indent=2, default=lambda o: o.tolist() if hasattr(o, "tolist") else o))
