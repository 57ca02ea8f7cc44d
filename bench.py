"""Benchmark: the plain tracer at scale (config 2), whole-job Mpaths/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 64 icospheres (Blender subdivisions 5) on a 512x512-cell fBm
terrain, 851,968 triangles, noise->ramp->mix Principled material per object,
1 sun + 16 point lights, 1920x1080, 64 spp, max depth 12, PCG32 seed 1.
A step renders one full 64-spp frame (132.7 M paths).  With N ranks every
rank renders its own 64 samples of the same image (sample ranges disjoint):
weak scaling, no collective inside the timed steps.  Afterwards the ranks'
films of their last step are summed into rank 0's renderer (one NCCL reduce
of the W x H float4 film on the devices, `frame` in the line), so rank 0
holds one image of all ranks' samples.

`value`  : paths of all ranks / max-over-ranks device time (CUDA events of
           the library's stream, reported by rmd_renderer_stats), scene and
           path pool resident.
`e2e`    : the same metric through the public C ABI with host buffers: each
           step uploads the camera (rmd_renderer_set_camera), renders and
           reads the film back to host memory (rmd_film_read).
`guided` : the learned path guide on the glossy room (config 4: 197,490
           triangles, lit through a 0.5 x 0.5 window, 1280x720, max depth 16):
           relMSE against an FP64 oracle of 65,536 spp of the plain tracer,
           plain tracer at 1,024 spp against the guided tracer (online
           training, 2^20 samples per Adam step, lr 1e-3) rendered in 32-spp
           chunks for up to 3x the plain tracer's device time: the guided
           tracer's time to the plain tracer's 1,024-spp relMSE and its relMSE
           at equal time.  Rank 0 only; --no-guided skips it.
--workload batch: config 3 instead: 64 independent config-2-style scenes
           (seed i, triangles log-uniform in [10k, 2M], resolution 2^U[7,10]
           squared) traced as one batch (one wavefront, one CUDA-graph
           launch per step), 32 spp, depth 10, autotuned; value = aggregate
           Mpaths/s, with each instance's paths and resolution in `instances`.
--workload config5: 16 glossy rooms tiled 4 x 4 (3.95 M triangles, metallic
           Bernoulli(0.5), 64 small emitters of radiance 500), 8 views in one
           batch, depth 20: plain batch at 1,024 spp against the guided batch
           (online training), relMSE per view against an FP64 oracle of
           --oracle-spp spp; at --c5-size per view (3840x2160 is the full
           size; the default is reduced to keep the oracle tractable).
--impl reference times the reference's own CPU implementation of the path
(its device code built for the host, oracle/_ref, all host cores; the oracle
restatement when that build is absent) on a bounded sample of the workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H, SPP, DEPTH, SEED = 1920, 1080, 64, 12, 1
WORKLOAD = "spheres_terrain_1080p_64spp_depth12"
METRIC = "Mpaths/s (plain tracer, config 2)"
# Algorithmic HBM bytes each stage must move per unit (queue-ordered path
# state, 16-byte records):
#   trace   per closest-hit ray: ray in (32), hit record out (16 + 4)
#   shade   per shaded segment : path state in (5 x 16 + hit 4), triangle
#           attributes (face 16, 3 x position 16, 3 x normal 16, 3 x uv 8),
#           continued path state out (5 x 16), shadow ray out (48)
#   shadow  per shadow ray     : ray + weight in (48), radiance read-modify-write (32)
#   film    per path           : finish record in (16), film read-modify-write (32),
#           new path state out (5 x 16)
BYTES_TRACE_PER_RAY = 32 + 20
BYTES_SHADE_PER_SEGMENT = 84 + 136 + 80 + 48
BYTES_SHADOW_PER_RAY = 48 + 32
BYTES_FILM_PER_PATH = 16 + 32 + 80
# DRAM bytes per unit measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum
# of one steady-state launch of the 480x270 case divided by the rays it
# processed); only the closest-hit kernel's is used
TRAFFIC_PER_UNIT = {"trace": 172.3}
# One segment (a closest-hit ray traced and shaded, with its NEE shadow ray) must move at least: ray in 32,
# hit written and read 20 + 20, path state read and written 32 + 32, next ray 32, hit-triangle attributes
# 110, shadow ray written 48, read by the shadow trace 32, occlusion flag written and read 8, shadow
# resolve read 16, film add 24.
BYTES_PER_SEGMENT = 406
GUIDED_W, GUIDED_H, GUIDED_DEPTH, GUIDED_ORACLE_SPP, GUIDED_PLAIN_SPP, GUIDED_CHUNK = 1280, 720, 16, 65536, 1024, 32
# guide settings of the guided legs (configs 4 and 5): Adam steps per 2^20 tracer samples, records per step
# the guided legs' training settings; the learning rate is three times the
# library's default (a sweep on the config-4 room measured it best)
GUIDE_DEFAULTS = {"batch_size": 1 << 20, "learning_rate": 3e-3, "steps_per_batch": 8, "step_records": 1 << 13}
CPU_BASELINE_SPP = 16  # CPU sample: 16 one-spp frames of the full image (about 10-20 s on 16 cores)


from raymond_b200.multi import (combine_films, max_over_ranks, rank_info, sample_range, shard_views,  # noqa: E402
                                sum_over_ranks)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows: list[list[str]] = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def make_scene():
    from raymond_b200 import scenes

    return scenes.spheres_terrain(seed=SEED)


class CpuReference:
    """The reference's own CPU implementation of the path when its host build is
    present (oracle/_ref/libref.so: the reference's kernels, lights, materials
    and envmap compiled for the host, all cores), else the oracle (the CPU
    restatement).  One call renders one 1-spp frame of the full image."""

    def __init__(self, desc):
        sys.path.insert(0, str(ROOT / "oracle"))
        sys.path.insert(0, str(ROOT / "oracle" / "ref"))
        import oracle_ctypes as O
        import ref_ctypes as R

        self.O = O
        self.orc = O.OracleScene(desc)
        self.ref = None
        if R.available():
            self.ref = R.RefScene(desc, "spheres_terrain", self.orc.surface_emissive())
        self.kind = "reference" if self.ref is not None else "port"

    def frame(self, k: int) -> dict:
        if self.ref is not None:
            film = self.ref.render(W, H, 1, DEPTH, sampling_mode=2, first_frame=k)
            return {"paths": W * H, "segments": None}
        _, st = self.orc.render(W, H, 1, DEPTH, first_sample=k, seed=SEED)
        return st

    def describe(self, frames: int) -> str:
        what = ("the reference's own kernels (host build of raymond/device: handleIntersections, raytrace, "
                "lights, envmap, node library; TEA generator)" if self.ref is not None
                else "the oracle (CPU restatement of the reference's integrator, PCG32)")
        return f"{frames} x 1 spp of the {W}x{H} frame (depth {DEPTH}) with {what} on {self.O.cpu_model()}"


def cpu_baseline_sample(desc):
    """CPU_BASELINE_SPP frames of the workload on all host cores."""
    ref = CpuReference(desc)
    t0 = time.perf_counter()
    paths = 0
    for k in range(CPU_BASELINE_SPP):
        paths += ref.frame(k)["paths"]
    dt = time.perf_counter() - t0
    return {"value": paths / dt / 1e6, "unit": "Mpaths/s", "cores": ref.O.cores(), "kind": ref.kind,
            "sample": ref.describe(CPU_BASELINE_SPP), "seconds": dt}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    from raymond_b200._abi import SceneDesc

    desc = SceneDesc(make_scene())
    ref = CpuReference(desc)
    # one step = 1 spp of the full frame (a bounded sample of the 64-spp step)
    for k in range(args.warmup):
        ref.frame(k)
    paths, secs = 0, 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        paths += ref.frame(k)["paths"]
        secs += time.perf_counter() - t0
    v = paths / secs / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpaths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "max_depth": DEPTH,
                       "step": "1 spp of the frame per step (bounded CPU sample)"},
            "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": ref.O.cores(), "kind": ref.kind,
                             "sample": ref.describe(args.steps)},
            "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


BATCH_INSTANCES, BATCH_SPP, BATCH_DEPTH = 64, 32, 10


def batch_instance(i: int, rng) -> tuple[dict, int, int]:
    """Config-2-style scene i with its triangle target and square resolution."""
    from raymond_b200 import scenes

    target = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
    res = 1 << int(rng.integers(7, 11))
    # 64 icospheres of 5 * 4^s faces take about half the triangles, the terrain the rest
    sub = max(1, min(6, int(np.floor(np.log(max(target / 2, 320) / 320) / np.log(4))) + 1))
    while sub > 1 and 64 * 5 * 4 ** sub > target / 2:
        sub -= 1
    cells = max(8, int(np.sqrt(max(target - 64 * 5 * 4 ** sub, 128) / 2)))
    sc = scenes.spheres_terrain(seed=i, subdivisions=sub, terrain_cells=cells, envmap_exponent=4)
    return sc, res, target


def run_batch(args, ctx=None, steps=None, warmup=None) -> dict:
    """Config 3: 64 scenes / views in one batch; returns the bench line."""
    from raymond_b200 import api, scenes
    from raymond_b200._abi import SceneDesc

    rank, world, local = rank_info()
    mine = set(shard_views(BATCH_INSTANCES, rank, world))  # instances of this rank (no exchange)
    rng = np.random.default_rng(3)
    t0 = time.perf_counter()
    descs, views, targets = [], [], []
    for i in range(BATCH_INSTANCES):
        sc, res, target = batch_instance(i, rng)  # every rank draws all, so instance i is the same everywhere
        if i not in mine:
            continue
        descs.append(SceneDesc(sc))
        views.append({"scene": len(descs) - 1, "width": res, "height": res})
        targets.append(target)
    ctx = ctx or api.Context(local)
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    b = api.Batch(ctx, descs, views)
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tune = b.autotune(spp=BATCH_SPP, max_depth=BATCH_DEPTH, seed=SEED)
    tune_s = time.perf_counter() - t0
    for k in range(warmup):
        b.reset()
        b.render(spp=BATCH_SPP, max_depth=BATCH_DEPTH, seed=SEED, first_sample=k * BATCH_SPP)
    sampler = ClockSampler(0)
    sampler.start()
    tot_ms, paths, segments = 0.0, 0, 0
    for k in range(steps):
        b.reset()
        b.render(spp=BATCH_SPP, max_depth=BATCH_DEPTH, seed=SEED, first_sample=k * BATCH_SPP)
        st = b.stats()
        tot_ms += st["ms_total"]
        paths += st["paths"]
        segments += st["segments"]
    clocks = sampler.stop()
    tris = [int(sum(len(s["indices"]) for s in d.scene["shapes"])) for d in descs]
    pixels = [v["width"] * v["height"] for v in views]
    tot_ms, = max_over_ranks([tot_ms])
    paths, segments = (int(x) for x in sum_over_ranks([float(paths), float(segments)]))
    value = paths / (tot_ms / 1e3) / 1e6
    line = {
        "metric": "Mpaths/s (batched, config 3)", "value": value, "unit": "Mpaths/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": tot_ms / steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes)",
        "config": {"workload": f"batch_{BATCH_INSTANCES}_instances_{BATCH_SPP}spp_depth{BATCH_DEPTH}",
                   "parallelism": f"{world} ranks x round-robin instances",
                   "instances": BATCH_INSTANCES, "total_pixels": sum(pixels), "total_triangles": sum(tris),
                   "launch": "one wavefront, one CUDA-graph launch per step (device-driven while loop)",
                   "l2": "inputs larger than L2 (path pool + BVHs + films)"},
        "msegments_per_s": segments / (tot_ms / 1e3) / 1e6,
        "instances": [{"triangles": t, "resolution": v["width"], "paths_per_step": p * BATCH_SPP,
                       "share_of_step_mpaths_per_s": p * BATCH_SPP / (tot_ms / steps / 1e3) / 1e6}
                      for t, v, p in zip(tris, views, pixels)],
        "clocks": clocks, "scene_build_s": build_s, "autotune": dict(tune, seconds=tune_s),
        "gpu_launches": steps,
    }
    b.close()
    return line


def run_config5(args) -> dict:
    """Config 5: guided + batched, 8 views of the 4 x 4 glossy rooms."""
    from raymond_b200 import api, scenes
    from raymond_b200._abi import SceneDesc
    from raymond_b200.metrics import relmse

    W, H = (int(x) for x in args.c5_size.split("x"))
    depth, chunk = 20, 32
    t0 = time.perf_counter()
    desc = SceneDesc(scenes.glossy_rooms_grid(seed=1))
    cams = scenes.grid_views(8)
    views = [{"scene": 0, "width": W, "height": H, "camera": c} for c in cams]
    ctx = api.Context(0)

    def batch():
        return api.Batch(ctx, [desc], views)
    oracle = batch()
    build_s = time.perf_counter() - t0
    per_call = max(1, min(args.oracle_spp, (1 << 27) // (W * H * 8)))
    done, oracle_ms = 0, 0.0
    while done < args.oracle_spp:
        n = min(per_call, args.oracle_spp - done)
        oracle.render(spp=n, max_depth=depth, film_fp64=True, seed=77)
        oracle_ms += oracle.stats()["ms_total"]
        done += n
    refs = [oracle.film64(v) / args.oracle_spp for v in range(8)]
    oracle.close()

    def errors(b):
        return [relmse(b.film(v, normalize=True), refs[v]) for v in range(8)]
    sampler = ClockSampler(0)
    sampler.start()
    plain = batch()
    plain_ms = 0.0
    for _ in range(GUIDED_PLAIN_SPP // chunk):
        plain.render(spp=chunk, max_depth=depth, seed=1)
        plain_ms += plain.stats()["ms_total"]
    e_plain = errors(plain)
    plain.close()
    g = batch()
    settings = dict(GUIDE_DEFAULTS)
    g.set_guide(sampling=True, training=True, seed=1, **settings)
    ms, spp, parity, curve = 0.0, 0, None, []
    target = float(np.mean(e_plain))
    while ms < 3 * plain_ms:
        g.render(spp=chunk, max_depth=depth, seed=2)
        ms += g.stats()["ms_total"]
        spp += chunk
        e = errors(g)
        curve.append((spp, ms, float(np.mean(e))))
        if parity is None and np.mean(e) <= target:
            parity = (spp, ms)
            break
    e_guided = errors(g)
    st = g.guide_stats()
    g.close()
    clocks = sampler.stop()
    return {
        "metric": "time to the plain tracer's 1024-spp relMSE, guided batch (config 5)",
        "clocks": clocks,
        "value": parity[1] / plain_ms if parity else None, "unit": "fraction of the plain batch's time",
        "value_interpolated": (crossing_ms(curve, target) / plain_ms) if parity else None,
        "higher_is_better": False, "n_gpus": 1,
        "config": {"workload": f"glossy_rooms_grid_4x4_8views_{W}x{H}_depth{depth}",
                   "triangles": desc_triangles(desc), "views": 8, "oracle_spp": args.oracle_spp,
                   "full_size": "3840x2160 per view", "reduced": (W, H) != (3840, 2160)},
        "oracle_device_s": oracle_ms / 1e3, "scene_build_s": build_s,
        "plain": {"spp": GUIDED_PLAIN_SPP, "ms": plain_ms, "relmse_per_view": e_plain, "relmse_mean": target},
        "guided": {"spp": spp, "ms": ms, "relmse_per_view": e_guided, "relmse_mean": float(np.mean(e_guided)),
                   "parity": {"spp": parity[0], "ms": parity[1]} if parity else None, "adam_steps": st["steps"],
                   "settings": settings,
                   "curve": [{"spp": a, "ms": round(b_, 1), "relmse": c} for a, b_, c in curve[::4]]},
    }


def desc_triangles(desc) -> int:
    return int(sum(len(s["indices"]) for s in desc.scene["shapes"]))


def crossing_ms(curve, target: float):
    """Time at which a relMSE curve [(spp, ms, relmse)] first reaches `target`,
    interpolated in log relMSE between the 32-spp chunks around the crossing
    (the chunk boundary itself quantises the time by up to a chunk)."""
    prev = None
    for s_, t_, e_ in curve:
        if e_ <= target:
            if prev is None or not (prev[2] > e_ > 0):
                return t_
            t0, e0 = prev[1], prev[2]
            return t0 + (t_ - t0) * (np.log(e0) - np.log(target)) / (np.log(e0) - np.log(e_))
        prev = (s_, t_, e_)
    return None


def guided_leg(api, ctx, oracle_spp: int, size=(GUIDED_W, GUIDED_H), guide: dict | None = None,
               oracle_cache: str = "") -> dict:
    """Equal-time relMSE of the guided tracer against the plain one (config 4).
    `guide` overrides the guide settings (GUIDE_DEFAULTS); `oracle_cache`, a
    .npy path: reuse the FP64 oracle film stored there by an earlier run of the
    same size and spp (its device time is then the stored run's)."""
    from raymond_b200 import scenes
    from raymond_b200._abi import SceneDesc
    from raymond_b200.metrics import relmse

    desc = SceneDesc(scenes.glossy_room(seed=1))
    scene = api.Scene(ctx, desc)
    (W, H), depth = size, GUIDED_DEPTH
    cache = Path(oracle_cache) if oracle_cache else None
    if cache and cache.exists():
        stored = np.load(cache, allow_pickle=True).item()
        assert stored["size"] == (W, H) and stored["spp"] == oracle_spp
        reference, oracle_ms = stored["film"], stored["ms"]
    else:
        oracle = api.Renderer(scene, W, H)
        per_call = max(1, min(oracle_spp, (1 << 27) // (W * H)))
        done, oracle_ms = 0, 0.0
        while done < oracle_spp:
            n = min(per_call, oracle_spp - done)
            oracle.render(spp=n, max_depth=depth, film_fp64=True, seed=77)
            oracle_ms += oracle.stats()["ms_total"]
            done += n
        reference = oracle.film64() / oracle_spp
        oracle.close()
        if cache:
            np.save(cache, {"size": (W, H), "spp": oracle_spp, "film": reference, "ms": oracle_ms})
    plain = api.Renderer(scene, W, H)
    plain_ms = 0.0
    for _ in range(GUIDED_PLAIN_SPP // GUIDED_CHUNK):
        plain.render(spp=GUIDED_CHUNK, max_depth=depth, seed=1)
        plain_ms += plain.stats()["ms_total"]
    e_plain = relmse(plain.film(normalize=True), reference)
    plain.close()
    settings = dict(GUIDE_DEFAULTS, **(guide or {}))
    g = api.Renderer(scene, W, H)
    g.set_guide(sampling=True, training=True, seed=1, **settings)
    ms, spp, curve, parity = 0.0, 0, [], None
    guide_ms = train_ms = 0.0
    while ms < 3 * plain_ms:
        g.render(spp=GUIDED_CHUNK, max_depth=depth, seed=2)
        st = g.stats()
        ms += st["ms_total"]
        guide_ms += st["ms_guide"]
        train_ms += st["ms_guide_train"]
        spp += GUIDED_CHUNK
        e = relmse(g.film(normalize=True), reference)
        curve.append((spp, ms, e))
        if parity is None and e <= e_plain:
            parity = (spp, ms)
        if parity is not None and ms >= plain_ms:  # both the parity time and the equal-time error are known
            break
    # relMSE at the plain tracer's time (interpolated between chunks)
    e_eq = None
    for (s0, t0, e0), (s1, t1, e1) in zip(curve, curve[1:]):
        if t0 <= plain_ms <= t1:
            e_eq = e0 + (e1 - e0) * (plain_ms - t0) / (t1 - t0)
    stats = g.guide_stats()
    g.close()
    return {
        "workload": f"glossy_room_{W}x{H}_depth{depth}", "triangles": scene.info()["triangles"],
        "oracle": {"spp": oracle_spp, "film": "fp64", "tracer": "plain", "device_s": oracle_ms / 1e3},
        "plain": {"spp": GUIDED_PLAIN_SPP, "ms": plain_ms, "relmse": e_plain},
        "guided": {"relmse_at_equal_time": e_eq, "ms_to_plain_relmse": parity[1] if parity else None,
                   "spp_to_plain_relmse": parity[0] if parity else None,
                   "time_ratio": parity[1] / plain_ms if parity else None, "target_time_ratio": 1.0 / 3.0,
                   "time_ratio_interpolated": (crossing_ms(curve, e_plain) / plain_ms) if parity else None,
                   "ms_guide": guide_ms, "ms_guide_train": train_ms, "adam_steps": stats["steps"],
                   "records": stats["records"], "settings": settings,
                   "curve": [{"spp": s_, "ms": round(t_, 2), "relmse": e_} for s_, t_, e_ in curve[::4]]},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pool", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--width", type=int, default=W, help="override (profiling runs only)")
    ap.add_argument("--height", type=int, default=H, help="override (profiling runs only)")
    ap.add_argument("--spp", type=int, default=SPP, help="override (profiling runs only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-guided", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--workload", default="plain", choices=["plain", "batch", "guided", "guided-render", "config5"])
    ap.add_argument("--c5-size", default="480x270", help="config 5: per-view resolution (full size 3840x2160)")
    ap.add_argument("--guided-size", default=f"{GUIDED_W}x{GUIDED_H}", help="guided leg resolution (profiling runs)")
    ap.add_argument("--oracle-spp", type=int, default=GUIDED_ORACLE_SPP, help="guided leg: oracle samples")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--guide-steps", type=int, default=0, help="--workload guided: Adam steps per batch")
    ap.add_argument("--guide-records", type=int, default=0, help="--workload guided: records per Adam step")
    ap.add_argument("--guide-batch", type=int, default=0, help="--workload guided: tracer samples per batch")
    ap.add_argument("--guide-lr", type=float, default=0.0, help="--workload guided: learning rate")
    ap.add_argument("--guide-depth", type=int, default=0, help="--workload guided: guided path depths (0: all)")
    ap.add_argument("--oracle-cache", default="", help="--workload guided: .npy file of the FP64 oracle film")
    ap.add_argument("--bvh", default="host", choices=["host", "gpu"], help="BVH builder of the plain workload's scene")
    ap.add_argument("--tuning", default="", help="shade_min_blocks,trace_blocks_per_sm,pool_size: apply "
                    "these launch choices instead of autotuning (profiling runs)")
    args = ap.parse_args()
    globals().update(W=args.width, H=args.height, SPP=args.spp)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        rank, world, _ = rank_info()
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        line = run_batch(args)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.workload == "config5":
        if args.oracle_spp == GUIDED_ORACLE_SPP:
            args.oracle_spp = 8192
        print(json.dumps(run_config5(args)), flush=True)
        return
    guided_size = tuple(int(x) for x in args.guided_size.split("x"))
    if args.workload == "guided-render":  # the guided tracer alone, --steps chunks of 32 spp (profiling runs)
        from raymond_b200 import api as api_, scenes
        from raymond_b200._abi import SceneDesc as SceneDesc_
        ctx_ = api_.Context(0)
        g = api_.Renderer(api_.Scene(ctx_, SceneDesc_(scenes.glossy_room(seed=1))), *guided_size)
        g.set_guide(sampling=True, training=True, seed=1, batch_size=1 << 20, learning_rate=1e-3)
        for _ in range(args.steps):
            g.render(spp=GUIDED_CHUNK, max_depth=GUIDED_DEPTH, seed=2)
        print(json.dumps({"workload": "guided-render", "stats": g.stats(), "guide": g.guide_stats()}), flush=True)
        return
    if args.workload == "guided":  # the config-4 leg alone
        from raymond_b200 import api as api_
        guide = {k: v for k, v in (("steps_per_batch", args.guide_steps), ("step_records", args.guide_records),
                                   ("batch_size", args.guide_batch), ("learning_rate", args.guide_lr),
                                   ("guided_depth", args.guide_depth)) if v}
        print(json.dumps(guided_leg(api_, api_.Context(0), args.oracle_spp, guided_size, guide, args.oracle_cache)),
              flush=True)
        return

    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist  # noqa: F811

        if torch.cuda.is_available():  # one rank per GPU: NCCL for the timing reductions and the film reduce
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device(f"cuda:{local}"))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))

    from raymond_b200 import api
    from raymond_b200._abi import SceneDesc, make_camera

    desc = SceneDesc(make_scene())
    ctx = api.Context(local, bvh_builder=args.bvh)
    t0 = time.perf_counter()
    scene = api.Scene(ctx, desc)
    build_s = time.perf_counter() - t0
    bvh = scene.bvh_stats()
    r = api.Renderer(scene, W, H, pool_size=args.pool)
    t0 = time.perf_counter()
    if args.tuning:
        mb, tb, pool = (int(x) for x in args.tuning.split(","))
        tune = {"shade_min_blocks": mb, "trace_blocks_per_sm": tb, "pool_size": pool, "applied": True}
        r.set_tuning(tune)
    else:
        tune = None if args.no_autotune else r.autotune(spp=SPP, max_depth=DEPTH, seed=SEED)
    tune_s = time.perf_counter() - t0
    cam = desc.scene["camera"]
    # the frame's host buffer in pinned memory (the device -> host read of every e2e step)
    try:
        import torch

        film_host = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True).numpy()
    except (ImportError, RuntimeError):
        film_host = np.zeros((H, W, 3), np.float32)

    def step(k, e2e=False):
        first, _ = sample_range(rank, world, k, SPP)
        if e2e:
            r.set_camera(cam)  # host -> device: camera
        else:
            r.reset()
        r.render(spp=SPP, max_depth=DEPTH, seed=SEED, first_sample=first)
        if e2e:
            r.film(out=film_host)  # device -> host: the frame
        return r.stats()

    for k in range(args.warmup):
        step(k)
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    tot_ms, tot = 0.0, {"paths": 0, "segments": 0, "rays": 0, "shadow_rays": 0, "iterations": 0, "ms_trace": 0.0,
                        "ms_shade": 0.0, "ms_shadow": 0.0, "ms_film": 0.0}
    for k in range(args.steps):
        s = step(k)
        tot_ms += s["ms_total"]
        for key in tot:
            tot[key] += s[key]
    clocks = sampler.stop()
    # end to end through the C ABI with host buffers
    t0 = time.perf_counter()
    for k in range(0 if args.no_e2e else args.steps):
        step(k, e2e=True)
    e2e_s = max(time.perf_counter() - t0, 1e-9)
    # the frame of all ranks: each rank's last step holds its own SPP samples of the image; the films
    # are summed into rank 0's renderer on the devices (NCCL reduce of W*H float4)
    t0 = time.perf_counter()
    frame_samples = combine_films(r)
    reduce_s = time.perf_counter() - t0
    if dist:
        tot_ms, e2e_s, reduce_s = max_over_ranks([tot_ms, e2e_s, reduce_s])
        dist.barrier()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    paths_all = tot["paths"] * world
    value = paths_all / (tot_ms / 1e3) / 1e6
    seg_rate = tot["segments"] * world / (tot_ms / 1e3)
    e2e_value = paths_all / e2e_s / 1e6
    stage_ms = {"film_regen": tot["ms_film"], "trace": tot["ms_trace"], "shade": tot["ms_shade"],
                "shadow": tot["ms_shadow"]}
    dominant = max(stage_ms, key=stage_ms.get)
    units = {"trace": (tot["rays"] + 0.0, BYTES_TRACE_PER_RAY),
             "shade": (tot["segments"] + 0.0, BYTES_SHADE_PER_SEGMENT),
             "shadow": (tot["shadow_rays"] + 0.0, BYTES_SHADOW_PER_RAY),
             "film_regen": (tot["paths"] + 0.0, BYTES_FILM_PER_PATH)}
    n_units, bpu = units[dominant]
    achieved = n_units * bpu / (stage_ms[dominant] / 1e3) / 1e9
    launches = max(1, tot["iterations"])  # one launch of each stage per iteration
    traffic = TRAFFIC_PER_UNIT[dominant] * n_units / launches if dominant in TRAFFIC_PER_UNIT else None
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    line = {
        "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD, "width": W, "height": H, "spp_per_rank_step": SPP, "max_depth": DEPTH,
                   "rng": "PCG32 seed 1", "triangles": scene.info()["triangles"],
                   "l2": "inputs larger than L2 (path pool + BVH + film)", "pool_size": r.stats()["pool_size"],
                   "parallelism": f"{world} ranks x disjoint sample ranges"},
        "segments_per_s": seg_rate, "msegments_per_s": seg_rate / 1e6,
        "mrays_per_s": tot["rays"] * world / (tot_ms / 1e3) / 1e6,
        "stage_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()},
        "iterations_per_step": tot["iterations"] / args.steps,
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": "measured" if peaks else "fallback",
                     "bytes_per_unit": bpu, "traffic": traffic,
                     "units_per_launch": n_units / launches},
        # the whole path's roofline by the per-segment definition: compulsory structure-of-arrays traffic
        # of one closest-hit ray traced and shaded with its shadow ray, at the measured segment rate
        "roofline_segment": {"bound": "hbm", "bytes_per_segment": BYTES_PER_SEGMENT,
                             "achieved": seg_rate * BYTES_PER_SEGMENT / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": seg_rate * BYTES_PER_SEGMENT / 1e9 / peak},
        "e2e": None if args.no_e2e else {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": 64 + 40,
                                         "d2h_bytes_per_step": W * H * 3 * 4},
        "gpu_launches": int(tot["iterations"] * 4 + args.steps),
        "frame": {"samples": frame_samples, "ranks": world, "reduce_ms": reduce_s * 1e3,
                  "reduce_bytes": W * H * 16 if world > 1 else 0,
                  "mean_radiance": float(r.film(normalize=True).mean())},
        "clocks": clocks,
        "scene_build_s": build_s, "bvh": bvh,
        "autotune": dict(tune, seconds=tune_s) if tune else None,
    }
    if not args.no_guided and world == 1:
        line["guided"] = guided_leg(api, ctx, args.oracle_spp, guided_size)
    if not args.no_batch and world == 1:
        bl = run_batch(args, ctx, steps=2, warmup=1)
        line["batched"] = {k: bl[k] for k in ("metric", "value", "unit", "ms_per_step", "msegments_per_s", "config",
                                              "autotune", "clocks", "scene_build_s")}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(desc)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
