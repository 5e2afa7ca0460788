"""Generate the converged references of the relMSE checks (test infrastructure).

For each workload, a seeded subset of pixels rendered by the oracle's FP64
plain path tracer (orc_render_f64: one RNG stream per (pixel, sample), the
workload's depth and clamp, Russian roulette on) at 16,384 spp.  The bench
computes relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + 0.01)
of its frames against these.  Run from the repository root:

    python tests/golden/make_relmse_refs.py [name ...]

Writes tests/golden/relmse_<name>.npz (pixels, ref, spp, seed).
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402
from raymotion_b200.scenes import cornell_box, icosphere_field  # noqa: E402

SPP = 16384
N_PIXELS = 4096


def workloads():
    def icosphere720():
        sb, cam, cfg = icosphere_field(seed=1)
        return sb.pack(), cam, cfg

    def cornell():
        sb, cam, cfg = cornell_box(0)
        return sb.pack(), cam, cfg

    return {"icosphere720": icosphere720, "cornell": cornell}


def make(name: str) -> Path:
    scene, cam, cfg = workloads()[name]()
    scene = pyoracle.with_reference_bvh(scene)
    npix = cfg.width * cfg.height
    pixels = np.sort(np.random.default_rng(2024).choice(npix, min(N_PIXELS, npix), replace=False)).astype(np.int32)
    cfg.spp = SPP
    t0 = time.time()
    ref = pyoracle.render_f64(scene, cam, cfg, 99991, pixels=pixels)
    out = Path(__file__).with_name(f"relmse_{name}.npz")
    np.savez_compressed(out, pixels=pixels, ref=ref, spp=SPP, seed=99991)
    print(f"{name}: {len(pixels)} pixels x {SPP} spp in {time.time() - t0:.0f} s -> {out.name}")
    return out


if __name__ == "__main__":
    pyoracle.build_oracle()
    for n in sys.argv[1:] or list(workloads()):
        make(n)
