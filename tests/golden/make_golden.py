"""Regenerate the oracle's golden fixtures (run from the repository root):

    python tests/golden/make_golden.py

prng.npz       PrngState.sample() streams (TEA and PCG32 bodies)
noise.npz      fractal_noise(p, detail 2, roughness 0.5) at 1024 seeded points
cornell_64.npz film sums of the 64x64 Cornell box, 4 samples, depth 8, PCG32 seed 1
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import oracle_ctypes as O  # noqa: E402
from raymond_b200 import scenes  # noqa: E402
from raymond_b200._abi import SceneDesc  # noqa: E402

OUT = Path(__file__).resolve().parent


def main():
    O.build()
    streams = {}
    for mode, a, b in [(0, 1, 0), (0, 1, 65537), (0, 42, 54), (1, 1, 0), (1, 7, 1234)]:
        streams[f"s_{mode}_{a}_{b}"] = O.prng(mode, a, b, 64)
    np.savez(OUT / "prng.npz", **streams)
    rng = np.random.default_rng(5)
    p = rng.uniform(-50, 50, (1024, 3)).astype(np.float32)
    np.savez(OUT / "noise.npz", p=p, v=O.fractal_noise3(p, 2.0, 0.5))
    orc = O.OracleScene(SceneDesc(scenes.cornell(seed=1, envmap_exponent=4)))
    film, st = orc.render(64, 64, 4, 8)
    np.savez_compressed(OUT / "cornell_64.npz", film=film, segments=st["segments"])


if __name__ == "__main__":
    main()
