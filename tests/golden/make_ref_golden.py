"""Regenerate tests/golden/ref_pin.npz from the host build of the reference's
own device code (oracle/_ref/libref.so, built by oracle/ref/Makefile from the
mounted reference).  Run from the repository root:

    make -C oracle/ref && python tests/golden/make_ref_golden.py [--only pin|render|tonemap|sky]

Contents: the reference's normalizeImage (exposure, accumulation, Hable and
ACES tonemaps) on a random film (ref_tonemap.npz); its Nishita sky model
(host/sky/sky_nishita.cpp) on small textures and the sun disc (ref_sky.npz);
TEA PRNG streams, fractal noise values and the evaluate/sample
results of every material in oracle/ref/pin_materials.py on seeded shading
records, all computed by the reference's code (ref_pin.npz); and one-sample
images of the reference-render scenes rendered by the reference's own kernels
(raytrace, handleIntersections, raytraceAny, handleShadowRays, the lights and
the environment map) in all three sampling modes (ref_render.npz).
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle" / "ref"))

sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))

import oracle_ctypes as O  # noqa: E402
import pin_materials  # noqa: E402
import ref_ctypes as R  # noqa: E402
from raymond_b200._abi import SceneDesc  # noqa: E402

PRNG_CASES = [(1, 0), (1, 77), (99, 4242), (123456, 7), (0xFFFFFFFF, 0xFFFFFFFF)]
NOISE_CASES = [(0.0, 0.5), (2.0, 0.5), (3.5, 0.7), (15.0, 1.0)]
RECORDS, RECORD_SEED = 512, 2024
# reference-render images: scene, width, height, max depth, first frames
RENDER_CASES = [("cornell", 48, 40, 8, [0, 5]), ("cornell_all_lights", 48, 40, 6, [0, 3]),
                ("spheres_small", 64, 36, 12, [0, 1])]
SAMPLING_MODES = [0, 1, 2]  # BSDF, NEE, MIS


# normalizeImage cases: exposure, accumulate, frame index, tonemapping (linear, Hable, ACES)
TONEMAP_CASES = [(e, a, f, t) for t in (0, 1, 2) for e, a, f in ((1.0, 0, 0), (1.7, 1, 0), (0.6, 1, 6))]


def tonemap_golden() -> None:
    """ref_tonemap.npz: the reference's normalizeImage kernel on a heavy-tailed
    random film (zeros, tiny and very large values included)."""
    rng = np.random.default_rng(11)
    film = (np.abs(rng.standard_cauchy((41, 29, 4))) * 3).astype(np.float32)
    film[0, :4] = [0, 1e-30, 1e20, 3e38]
    out = {"film": film, "cases": np.array(TONEMAP_CASES, np.float32),
           "images": np.stack([R.normalize_image(film, e, bool(a), int(f), int(t)) for e, a, f, t in TONEMAP_CASES])}
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_tonemap.npz", **out)


# Nishita sky cases: sun elevation, altitude, air, dust, ozone (the texture) and sun rotation, size, intensity
SKY_CASES = [(0.2618, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0095, 1.0), (0.05, 1000.0, 2.0, 0.5, 1.0, 1.3, 0.2, 2.0),
             (-0.1, 0.0, 1.0, 1.0, 1.0, 4.0, 0.05, 1.0), (1.2, 5e4, 0.3, 4.0, 2.0, 0.5, 0.6, 0.5)]
SKY_SIZE = 64  # texture width and height of the golden (the renderer's is 512)


def sky_golden() -> None:
    """ref_sky.npz: the reference's sky model (host/sky/sky_nishita.cpp) on a
    64 x 64 texture and the sun disc colours, for each case."""
    tex, sun = [], []
    for e, alt, air, dust, oz, _rot, size, _inten in SKY_CASES:
        tex.append(R.sky_texture(SKY_SIZE, SKY_SIZE, e, alt, air, dust, oz))
        sun.append(R.sky_sun(e, size, alt, air, dust))
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_sky.npz", cases=np.array(SKY_CASES, np.float32),
                        textures=np.stack(tex), sun=np.stack(sun))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["pin", "render", "tonemap", "sky"], help="regenerate one file")
    args = ap.parse_args()
    if args.only in (None, "tonemap"):
        tonemap_golden()
    if args.only in (None, "sky"):
        sky_golden()
    if args.only in (None, "pin"):
        pin_golden()
    if args.only in (None, "render"):
        render_golden()


def pin_golden() -> None:
    out = {}
    out["prng_cases"] = np.array(PRNG_CASES, np.uint64)
    out["prng"] = np.stack([R.prng_tea(a, b, 256) for a, b in PRNG_CASES])
    rng = np.random.default_rng(5)
    pts = rng.uniform(-50, 50, (2048, 3)).astype(np.float32)
    out["noise_points"] = pts
    out["noise_cases"] = np.array(NOISE_CASES, np.float32)
    out["noise"] = np.stack([R.fractal_noise3(pts, d, r) for d, r in NOISE_CASES])
    pin_materials.install_ref_textures(R)
    rec = R.shading_records(RECORDS, RECORD_SEED)
    names = [n for n, _ in pin_materials.materials()]
    out["records"] = rec
    out["material_names"] = np.array(names)
    out["materials"] = np.stack([R.material_eval(m, rec) for m in range(len(names))])
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_pin.npz", **out)


def render_golden() -> None:
    scenes = pin_materials.ref_scenes()
    renders = {}
    for name, w, h, depth, frames in RENDER_CASES:
        desc = SceneDesc(scenes[name])
        ref = R.RefScene(desc, name, O.OracleScene(desc).surface_emissive())
        renders[f"{name}/size"] = np.array([w, h, depth], np.int32)
        for mode in SAMPLING_MODES:
            for f in frames:
                renders[f"{name}/{mode}/{f}"] = ref.render(w, h, 1, depth, sampling_mode=mode, first_frame=f)
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_render.npz", **renders)


if __name__ == "__main__":
    main()
