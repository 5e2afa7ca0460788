"""Generate the converged references of the relMSE checks (test infrastructure).

For each workload, a seeded subset of pixels rendered by the oracle's FP64
plain path tracer (orc_render_f64: one RNG stream per (pixel, sample), the
workload's depth, clamp and Russian-roulette setting: on for the icosphere
field, off for the Cornell box as config 0 states) at 16,384 spp.  The bench
computes relMSE = mean over pixels and channels of (I - R)^2 / (R^2 + 0.01)
of its frames against these.  Run from the repository root:

    python tests/golden/make_relmse_refs.py [name ...]

Writes tests/golden/relmse_<name>.npz (pixels, ref, spp, seed); the batched
workload's 64 scenes go to relmse_batch.npz (scene, pixels, ref, spp).
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402
from raymotion_b200 import objects  # noqa: E402
from raymotion_b200.scenes import AnimatedSequence, batch_workload, cornell_box, icosphere_field, sized_field  # noqa: E402

SPP = 16384
N_PIXELS = 4096


def workloads():
    def icosphere720():
        sb, cam, cfg = icosphere_field(seed=1)
        return sb.pack(), cam, cfg

    def cornell():
        sb, cam, cfg = cornell_box(0)
        return sb.pack(), cam, cfg

    def sequence33():
        # the animated sequence's last frame (frame 33: cloth, moving spheres and camera at t = 33 / 30 s)
        seq = AnimatedSequence()
        models = list(seq.models)
        models[seq.CLOTH] = seq.cloth(33)
        world = objects.world_builder(models, seq.instances(33)).pack()
        return world, seq.camera(33), seq.cfg

    return {"icosphere720": icosphere720, "cornell": cornell, "sequence33": sequence33}


BATCH_PIXELS = 256
BATCH_SPP = 8192


def make_batch() -> Path:
    """Per-scene references of the batched workload (64 scenes of
    batch_workload(seed=3)): BATCH_PIXELS seeded pixels of each image at
    BATCH_SPP spp, same depth, clamp and Russian roulette as the image."""
    specs = batch_workload(seed=3, n_scenes=64)
    rng = np.random.default_rng(2025)
    scene_idx, pixels, refs = [], [], []
    t0 = time.time()
    for k, sp in enumerate(specs):
        sb, cam, cfg = sized_field(**sp)
        scene = pyoracle.with_reference_bvh(sb.pack())
        npix = cfg.width * cfg.height
        pix = np.sort(rng.choice(npix, BATCH_PIXELS, replace=False)).astype(np.int32)
        cfg.spp = BATCH_SPP
        refs.append(pyoracle.render_f64(scene, cam, cfg, 99991 + k, pixels=pix))
        pixels.append(pix)
        scene_idx.append(np.full(len(pix), k, np.int32))
    out = Path(__file__).with_name("relmse_batch.npz")
    np.savez_compressed(out, scene=np.concatenate(scene_idx), pixels=np.concatenate(pixels),
                        ref=np.concatenate(refs), spp=BATCH_SPP)
    print(f"batch: 64 scenes x {BATCH_PIXELS} pixels x {BATCH_SPP} spp in {time.time() - t0:.0f} s -> {out.name}")
    return out


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
    for n in sys.argv[1:] or list(workloads()) + ["batch"]:
        if n == "batch":
            make_batch()
        else:
            make(n)
