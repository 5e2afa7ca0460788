#!/usr/bin/env python
"""Benchmark: path samples/s of one raymotion frame on the B200 backend.

Workload (one "step" = one frame): the instanced icosphere field of
raymotion_b200.scenes.icosphere_field - 200 displaced icospheres + ground +
4096 small emitters = 1,028,098 triangles - rendered at 1280x720, 64 spp,
max depth 12, ReSTIR DI on (32 RIS candidates, 5 spatial neighbours within
30 px, temporal reuse from the previous frame) and the denoiser on; seeded
synthetic data (no dataset exists for this path).  The scene (181 MB of
triangles + 49 MB of traversal records) is larger than the 126 MB L2.

Reported on one JSON line (rank 0):
  value   - path samples/s with the scene resident in HBM, timed with CUDA
            events on the rendering stream over exactly --steps frames
            (max over ranks; each rank renders its own frames: replicas);
  e2e     - the same metric through the reference-facing call
            rmcuda_render with host buffers: scene upload from pinned host
            memory, device BVH build, frame, RGB8 read-back, every step;
  roofline- the dominant kernel (by summed CUDA-event time): algorithmic bytes
            it fetches (BVH records 64 B x nodes visited + triangle records
            48 B x tests, counted on the device) / its average launch time,
            against the measured HBM copy bandwidth;
  cpu_baseline - the CPU oracle (a restatement of the reference's Metal
            kernels; the reference itself runs only on Apple GPUs) timed on a
            band of rows of the same frame with every host core;
  batch   - batched vs one-at-a-time path samples/s over 64 uneven scenes
            (see batch_compare), with the images checked identical;
  adjoint - the path-replay adjoint's cost relative to the forward frame and
            a 200-step material fit (see adjoint_measure).
--impl reference times that CPU implementation alone.
"""
from __future__ import annotations

import argparse
import dataclasses
import datetime
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

METRIC = "path samples/s"
UNIT = "path samples/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="icosphere720", choices=["icosphere720", "icosphere180", "cornell"],
                    help="icosphere180: the same scene at 320x180, 16 spp (profiling size)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-step-seconds", type=float, default=None,
                    help="--impl reference: CPU seconds per step (default: about a minute over all steps)")
    ap.add_argument("--no-breakdown", action="store_true", help="skip the per-kernel timing frame")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-serial measurement")
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--no-sequence", action="store_true", help="skip the animated-sequence measurement")
    ap.add_argument("--no-relmse", action="store_true", help="skip the relMSE frames")
    ap.add_argument("--no-large", action="store_true", help="skip the 2048x1280 screen-space frames")
    ap.add_argument("--screen-space-only", action="store_true",
                    help="only the 2048x1280 screen-space frames (profiling the denoiser passes)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-rendering measurement")
    ap.add_argument("--fit-iters", type=int, default=200)
    return ap.parse_args()


def workload(name: str):
    from raymotion_b200.scenes import cornell_box, icosphere_field
    if name == "cornell":
        sb, cam, cfg = cornell_box(0)
        desc = dict(workload="cornell box, 36 triangles, 320x180, 16 spp, depth 8, plain NEE+MIS", triangles=36)
    elif name == "icosphere180":
        sb, cam, cfg = icosphere_field(seed=1, width=320, height=180, spp=16)
        desc = dict(workload="icosphere field, 1,028,098 triangles, 320x180, 16 spp, depth 12, ReSTIR DI "
                             "(32 candidates, 5 spatial neighbours, radius 30 px, temporal) + denoiser")
    else:
        sb, cam, cfg = icosphere_field(seed=1)
        desc = dict(workload="icosphere field, 1,028,098 triangles, 1280x720, 64 spp, depth 12, ReSTIR DI "
                             "(32 candidates, 5 spatial neighbours, radius 30 px, temporal) + denoiser")
    scene = sb.pack()
    desc.update(triangles=int(scene.n_tris), width=cfg.width, height=cfg.height, spp=cfg.spp,
                max_depth=cfg.max_bounces, l2="inputs larger than L2 (scene 181 MB + 49 MB BVH leaf records)",
                bvh="device PLOC BVH (leaves of at most 4 triangles)")
    return scene, cam, cfg, desc


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if not self.proc:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if len(r) >= 7 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 7 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 7 for k in range(4) if r[3 + k] == "Active"})
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(sm))


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
        except Exception:
            pass
    return dict(hbm_gbs=6650.0, source="fallback")


def ncu_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary, scaled to this workload."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return float(d[kernel]["dram_bytes_per_launch_full"])
    except Exception:
        return None


def rank_launch_command(argv: list[str], n: int, port: int) -> list[str]:
    """torch.distributed.run over n local ranks, rendezvous on 127.0.0.1, running
    this file with the same arguments (one process per GPU)."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
            "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *argv]


def launch_ranks(args, argv: list[str]) -> int:
    """bench.py --gpus N started without a launcher: start the N ranks here."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    return subprocess.run(rank_launch_command(argv, args.gpus, port)).returncode


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)  # each rank's communicator on its own GPU
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allreduce(values: list[float], op: str, world: int, device=None) -> list[float]:
    if world <= 1:
        return values
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return t.tolist()


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- CPU (oracle)

def cpu_band(scene, cam, cfg, seconds: float, rows_hint: int | None = None):
    """Time the CPU oracle on a band of rows of the same frame; returns (samples/s, desc, threads)."""
    from oracle import pyoracle
    if scene.nodes is None:
        pyoracle.with_reference_bvh(scene)
    o = pyoracle.Oracle()
    threads = pyoracle.nthreads()
    y0 = cfg.height // 2
    rows = rows_hint or 1
    # calibrate on one row, then size the band to the time budget
    if rows_hint is None:
        t0 = time.perf_counter()
        o.render(scene, cam, cfg, 777, threads=threads, rows=(y0, y0 + 1))
        dt = max(time.perf_counter() - t0, 1e-3)
        rows = int(max(1, min(cfg.height - y0, seconds / dt)))
        rows = max(rows, min(threads, cfg.height - y0))
    t0 = time.perf_counter()
    _, _, st = o.render(scene, cam, cfg, 778, threads=threads, rows=(y0, y0 + rows))
    dt = time.perf_counter() - t0
    return st["path_samples"] / dt, f"rows {y0}..{y0 + rows - 1} of the frame ({rows * cfg.width} pixels, " \
                                     f"{st['path_samples']} path samples, {dt:.1f} s)", threads, rows, dt


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    scene, cam, cfg, desc = workload(args.workload)
    per_step = args.ref_step_seconds or max(2.0, 60.0 / max(1, args.steps + args.warmup))
    _, _, threads, rows, _ = cpu_band(scene, cam, cfg, per_step)
    for _ in range(args.warmup):
        cpu_band(scene, cam, cfg, per_step, rows_hint=rows)
    vals, tsum = [], 0.0
    sample_desc = ""
    for _ in range(args.steps):
        v, sample_desc, threads, rows, dt = cpu_band(scene, cam, cfg, per_step, rows_hint=rows)
        vals.append(v)
        tsum += dt
    value = float(np.mean(vals))
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * tsum / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f32", data="synthetic (seeded procedural scene)", impl="reference",
                config=dict(desc, parallelism="cpu threads"),
                cpu_baseline=dict(value=value, unit=UNIT, cores=threads, kind="port",
                                  sample=f"per step: {sample_desc}"),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU

def batch_compare(args, backend, torch, stream, dev, world):
    """Batched vs one-at-a-time rendering of the uneven multi-scene workload.

    Scenes as raymotion_b200.scenes.batch_workload (seed 3): triangle counts
    log-uniform over [1k, 2M], resolutions from {256x256, 640x360, 1280x720,
    1920x1080}, spp from {4, 16, 64}, depth 8-12, plain path.  Serial: the
    single-frame policy per scene object (rmcuda_render_scene_async), all
    enqueued back to back; batched: rmcuda_render_batch with the settings
    rmcuda_batch_tune picked (tuning is untimed).  Both produce the same
    images bit for bit (checked), so their relMSE is equal."""
    from raymotion_b200 import BatchItem
    from raymotion_b200.scenes import batch_workload, sized_field
    from raymotion_b200.shard import rank_items
    all_specs = batch_workload(seed=3, n_scenes=args.batch_scenes)
    # with several ranks each renders a disjoint, cost-balanced subset of the
    # images (no data-path collective); one rank renders them all
    rank = int(os.environ.get("RANK", "0")) if world > 1 else 0
    mine = rank_items(all_specs, rank, world)
    specs = [all_specs[i] for i in mine]
    t0 = time.time()
    items, hdrs, handles = [], [], []
    for sp in specs:
        sb, cam, cfg = sized_field(**sp)
        h = backend.scene_create(sb.pack())
        handles.append(h)
        npix = cfg.width * cfg.height
        rgb = torch.empty(npix * 3, dtype=torch.uint8, device=dev)
        hdr = torch.empty(npix * 3, dtype=torch.float32, device=dev)
        hdrs.append((rgb, hdr))
        items.append(BatchItem(h, cam, cfg, 777, rgb.data_ptr(), hdr.data_ptr(), None))
    build_s = time.time() - t0

    def serial():
        for it in items:
            backend.render_scene_async(it.scene, it.camera, it.config, it.seed, it.d_rgb, it.d_hdr)

    def batched():
        backend.render_batch(items)

    def timed(fn):
        backend.stats_reset()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.batch_steps):
            fn()
        e1.record(stream)
        backend.sync()
        torch.cuda.synchronize()
        sec, = allreduce([e0.elapsed_time(e1) / 1e3], "max", world, dev)
        samples, = allreduce([float(backend.stats()["path_samples"])], "sum", world, dev)
        return sec, samples

    serial()
    backend.sync()
    ref = [h.clone() for _, h in hdrs]
    t1 = time.time()
    tuning = backend.batch_tune(items)
    tune_s = time.time() - t1
    batched()
    identical = all(torch.equal(h.view(torch.int32), r.view(torch.int32)) for (_, h), r in zip(hdrs, ref))
    s_sec, s_samples = timed(serial)
    b_sec, b_samples = timed(batched)
    s_own, = allreduce([float(sum(r[1].numel() for r in hdrs))], "sum", world, dev)  # every image rendered once
    # per-scene relMSE against the FP64 references (the batched images; the
    # serial ones are identical, checked above)
    rel = []
    g = ROOT / "tests" / "golden" / "relmse_batch.npz"
    if g.exists() and len(all_specs) == 64:
        ref = np.load(g)
        for k, gi in enumerate(mine):
            sel = ref["scene"] == gi
            img = hdrs[k][1].cpu().numpy().reshape(-1, 3)[ref["pixels"][sel]].astype(np.float64)
            rel.append(_relmse(img, ref["ref"][sel]))
    rel_sum, rel_n, rel_max = allreduce([float(sum(rel)), float(len(rel))], "sum", world, dev) + \
        allreduce([max(rel) if rel else 0.0], "max", world, dev)
    identical, = allreduce([1.0 if identical else 0.0], "sum", world, dev)
    log = backend.batch_log()
    for h in handles:
        backend.scene_destroy(h)
    return dict(
        workload=f"{len(all_specs)} seeded icosphere-field scenes, triangles log-uniform in [1k, 2M], resolutions "
                 "{256x256, 640x360, 1280x720, 1920x1080}, spp {4, 16, 64}, depth 8-12, plain path",
        triangles=int(sum(sp["n_tris"] for sp in all_specs)),
        pixels=int(sum(sp["width"] * sp["height"] for sp in all_specs)),
        sharding=dict(ranks=world, images_per_rank=len(mine), rank0_images=mine if rank == 0 else None,
                      pixels_rendered=int(s_own / 3), collective="none (timings and counts reduced only)"),
        steps=args.batch_steps, path_samples_per_step=int(b_samples / args.batch_steps),
        serial=dict(value=s_samples / s_sec, unit=UNIT, ms_per_step=1e3 * s_sec / args.batch_steps),
        batched=dict(value=b_samples / b_sec, unit=UNIT, ms_per_step=1e3 * b_sec / args.batch_steps,
                     tuning=tuning, progress_checks=int(len(log))),
        speedup=(b_samples / b_sec) / (s_samples / s_sec), identical_images=bool(identical == world),
        relmse=dict(scenes=int(rel_n), pixels_per_scene=256, ref_spp=8192, mean=rel_sum / rel_n, max=rel_max,
                    rank0_per_scene=[round(x, 5) for x in rel] if rank == 0 else None,
                    note="batched = serial per scene (identical images)") if rel_n else None,
        equal_samples=bool(s_samples == b_samples), scene_build_s=build_s, tune_s=tune_s)


def adjoint_measure(args, backend, torch, stream, dev, rank=0, world=1):
    """Differentiable rendering on raymotion_b200.scenes.inverse_scene: 100
    displaced icospheres (subdivision 3) + a 190 x 190-quad ground + 16 quad
    lights = 200,232 triangles, 256 materials, 512 x 512, 32 spp, depth 8.

    (1) forward frame vs rmcuda_backward, each timed with CUDA events over 3
    calls after 2 warm-ups: the adjoint/forward time ratio;  (2) the fit: a
    1024-spp target at the true materials, a start with +-30 % uniform noise on
    every fitted parameter (albedo and roughness of all materials, emission of
    the 16 lights, IOR of the 32 dielectrics), 200 Adam steps (lr 1e-2 on
    parameters normalised to their ranges) of an L2 loss at 32 spp, the adjoint
    replaying an independent frame each step (an unbiased gradient of the
    expected loss).  Reports the mean normalised parameter error before and
    after, over all fitted parameters and over those of materials the camera
    sees directly on at least 256 pixels.  With several ranks the fit is data
    parallel (raymotion_b200.inverse.MaterialFit): each rank renders its own
    seeds and the gradients are averaged by one all-reduce per step."""
    from raymotion_b200.inverse import MaterialFit
    import raymotion_b200 as rb
    from raymotion_b200.scene import with_materials
    from raymotion_b200.scenes import INVERSE_HI, INVERSE_LO, inverse_scene
    d = inverse_scene()
    sc, cam, cfg, tm = d["scene"], d["camera"], d["config"], d["tri_material"]
    n_mat = len(d["params"])
    h = backend.scene_create(sc)
    npix = cfg.width * cfg.height

    def set_params(p):
        s2 = with_materials(sc, tm, p)
        backend.scene_set_materials(h, p, tm, s2.light_cdf, s2.light_total)

    set_params(d["params"])
    img = torch.empty(npix * 3, dtype=torch.float32, device=dev)
    dl = torch.full((npix * 3,), 1e-6, dtype=torch.float32, device=dev)
    grad = torch.zeros(n_mat * 8, dtype=torch.float32, device=dev)

    def fwd(seed):
        backend.render_scene_async(h, cam, cfg, seed, None, img.data_ptr())

    def bwd(seed):
        backend.backward(h, cam, cfg, seed, dl.data_ptr(), grad.data_ptr())

    def timed(fn, k=3):
        for i in range(2):
            fn(100 + i)
        backend.sync()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(k):
            fn(200 + i)
        e1.record(stream)
        backend.sync()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    backend.stats_reset()
    fwd_ms = timed(fwd)
    bwd_ms = timed(bwd)
    st = backend.stage_counters()
    # the ReSTIR chain on the same scene: each adjoint replays the frame just
    # rendered (its G-buffer and reservoirs are the checkpoint)
    restir = dict(workload="the same scene and 32 spp on the ReSTIR chain (32 candidates, 5 neighbours, radius 30 "
                           "px, temporal); the adjoint replays K5 from the frame's G-buffer and reservoirs, and "
                           "transposes the denoiser when it is on")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for name, denoise in (("denoiser_off", False), ("denoised", True)):
        cfg_r = rb.RenderConfig(**{k: getattr(cfg, k) for k in cfg.__dataclass_fields__})
        cfg_r.restir_candidates, cfg_r.restir_spatial, cfg_r.restir_radius = 32, 5, 30.0
        cfg_r.flags = cfg.flags & ~rb._abi.RM_FLAG_RESTIR_OFF & ~rb._abi.RM_FLAG_DENOISE_OFF
        if not denoise:
            cfg_r.flags |= rb._abi.RM_FLAG_DENOISE_OFF
        r_fwd = r_bwd = 0.0
        for i in range(5):
            ev[0].record(stream)
            backend.render_scene_async(h, cam, cfg_r, 300 + i, None, img.data_ptr())
            ev[1].record(stream)
            backend.backward(h, cam, cfg_r, 300 + i, dl.data_ptr(), grad.data_ptr())
            ev[2].record(stream)
            backend.sync()
            torch.cuda.synchronize()
            if i >= 2:
                r_fwd += ev[0].elapsed_time(ev[1]) / 3
                r_bwd += ev[1].elapsed_time(ev[2]) / 3
        restir[name] = dict(forward_ms=r_fwd, adjoint_ms=r_bwd, adjoint_over_forward=r_bwd / r_fwd)
    # which materials the camera sees: primary hits of the pixel centres
    backend.upload(sc, use_nodes=False)
    ys, xs = np.mgrid[0:cfg.height, 0:cfg.width]
    sx = (xs + 0.5 - cfg.width * 0.5).astype(np.float32).ravel()
    sy = (cfg.height * 0.5 - (ys + 0.5)).astype(np.float32).ravel()
    f = np.float32(cam.focal)
    inv = np.float32(1) / np.sqrt(sx * sx + (sy * sy + f * f))
    m = np.asarray(cam.m, np.float32)
    tx, ty, tz = sx * inv, sy * inv, f * inv
    rays = np.zeros((npix, 7), np.float32)
    rays[:, 0:3] = (cam.x, cam.y, cam.z)
    rays[:, 3] = tx * m[0] + (ty * m[1] + tz * m[2])
    rays[:, 4] = tx * m[3] + (ty * m[4] + tz * m[5])
    rays[:, 5] = tx * m[6] + (ty * m[7] + tz * m[8])
    rays[:, 6] = 1e30
    d_rays = torch.from_numpy(rays).to(dev)
    d_tri = torch.empty(npix, dtype=torch.int32, device=dev)
    backend.trace(d_rays.data_ptr(), npix, False, d_tri.data_ptr())
    tri = d_tri.cpu().numpy()
    seen = np.bincount(tm[tri[tri >= 0]], minlength=n_mat) >= 256
    # the fit
    lo = torch.from_numpy(INVERSE_LO).to(dev)
    hi = torch.from_numpy(INVERSE_HI).to(dev)
    mask = torch.from_numpy(d["mask"]).to(dev)
    true = torch.from_numpy(d["params"]).to(dev)
    cfg_t = rb.RenderConfig(**{k: getattr(cfg, k) for k in cfg.__dataclass_fields__})
    cfg_t.spp = 1024
    backend.render_scene_async(h, cam, cfg_t, 1, None, img.data_ptr())
    backend.sync()
    target = img.clone()
    gen = torch.Generator(device=dev).manual_seed(4)
    noise = (torch.rand(true.shape, device=dev, generator=gen) * 2 - 1) * 0.3
    start = torch.where(mask, torch.minimum(torch.maximum(true * (1 + noise), lo), hi), true)
    fit = MaterialFit(start, true, mask, lo, hi, lr=1e-2)
    seen_t = torch.from_numpy(seen).to(dev)[:, None] & mask
    # metallic materials (their roughness shapes the whole lobe; a dielectric-free
    # non-metal's roughness only shapes its 4 % specular part)
    metal = np.zeros(n_mat, bool)
    np.logical_or.at(metal, tm, sc.tris["metallic"] > 0.5)
    metal_t = torch.from_numpy(metal).to(dev)

    def errors(p):
        e = (p - true).abs() / (hi - lo)
        out = dict(all=e[mask].mean().item(), seen=e[seen_t].mean().item() if seen_t.any() else None)
        for name, cols in (("albedo", slice(0, 3)), ("rough", slice(3, 4)), ("emission", slice(4, 7)),
                           ("ior", slice(7, 8))):
            mk = mask[:, cols]
            out[name] = e[:, cols][mk].mean().item() if mk.any() else None
            ms = mk & seen_t[:, cols]
            out[name + "_seen"] = e[:, cols][ms].mean().item() if ms.any() else None
        for name, sel in (("rough_seen_metal", metal_t), ("rough_seen_nonmetal", ~metal_t)):
            ms = mask[:, 3] & seen_t[:, 3] & sel
            out[name] = e[:, 3][ms].mean().item() if ms.any() else None
        return out

    err0 = errors(start)
    t0 = time.time()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    losses = []
    for it in range(args.fit_iters):
        set_params(fit.params().cpu().numpy())
        backend.render_scene_async(h, cam, cfg, 10000 + it + 1000003 * rank, None, img.data_ptr())
        dl.copy_((2.0 / img.numel()) * (img - target))
        losses.append(((img - target) ** 2).mean())
        grad.zero_()
        backend.backward(h, cam, cfg, 20000 + it + 1000003 * rank, dl.data_ptr(), grad.data_ptr())
        backend.sync()
        fit.step(grad)  # with several ranks: the mean gradient (one all-reduce)
    f1.record(stream)
    backend.sync()
    torch.cuda.synchronize()
    fit_s = time.time() - t0
    err1 = errors(fit.params())
    # image-space recovery: the start and fitted materials rendered at the
    # target's 1024 spp (another seed), relMSE against the target
    img_rel = {}
    for name, prm in (("start", start), ("fitted", fit.params())):
        set_params(prm.cpu().numpy())
        backend.render_scene_async(h, cam, cfg_t, 2, None, img.data_ptr())
        backend.sync()
        a = img.cpu().numpy().astype(np.float64)
        b = target.cpu().numpy().astype(np.float64)
        img_rel[name] = _relmse(a, b)
    set_params(d["params"])
    backend.render_scene_async(h, cam, cfg_t, 2, None, img.data_ptr())
    backend.sync()
    img_rel["true_other_seed"] = _relmse(img.cpu().numpy().astype(np.float64), target.cpu().numpy().astype(np.float64))
    backend.scene_destroy(h)
    loss_curve = [float(x) for x in torch.stack(losses).cpu().numpy()]
    return dict(
        workload="inverse_scene: 200,232 triangles, 256 materials, 512x512, 32 spp, depth 8, plain path, "
                 "fixed spp, Russian roulette on",
        forward_ms=fwd_ms, adjoint_ms=bwd_ms, adjoint_over_forward=bwd_ms / fwd_ms,
        adjoint_samples_per_call=int(st["adjoint"]["path_samples"] / 5), restir=restir,
        fit=dict(iterations=args.fit_iters, lr=1e-2, optimiser="Adam on normalised parameters",
                 target_spp=1024, fit_spp=cfg.spp, ranks=world, wall_s=fit_s, gpu_ms=f0.elapsed_time(f1),
                 param_error_start=err0, param_error_end=err1, materials_seen=int(seen.sum()),
                 relmse_1024spp_vs_target=img_rel,
                 loss_first10=float(np.mean(loss_curve[:10])), loss_last10=float(np.mean(loss_curve[-10:]))))


def sequence_measure(args, backend, torch, stream, dev):
    """The animated sequence: 34 frames at 1280x720, 16 spp, temporal ReSTIR and
    denoise on animated geometry (RM_FLAG_ANIMATED_HISTORY).  Per frame: the
    cloth model's new triangles uploaded (rmcuda_model_update, 36 MB from host
    memory), the world of 203 instances built on the device with the BVH
    refitted, or rebuilt every 32nd commit (rmcuda_instances_commit), and the
    frame rendered (rmcuda_render_resident_async).  The cloth frames are
    generated before the timed loop (the animation itself is the caller's).
    value = path samples over the sequence / its wall time, measured with CUDA
    events around the whole loop on the rendering stream.
    """
    import raymotion_b200 as rb
    from raymotion_b200 import objects
    from raymotion_b200.scenes import AnimatedSequence
    seq = AnimatedSequence()
    cfg = seq.cfg
    cloth = [seq.cloth(f) for f in range(seq.frames)]
    recs = [objects.instance_records(seq.instances(f)) for f in range(seq.frames)]
    cams = [seq.camera(f) for f in range(seq.frames)]
    ids = [backend.model_create(m) for m in seq.models]
    for r in recs:
        r["model"] = np.asarray(ids, np.int32)[r["model"]]
    npix = cfg.width * cfg.height
    d_rgb = torch.empty(npix * 3, dtype=torch.uint8, device=dev)
    d_hdr = torch.empty(npix * 3, dtype=torch.float32, device=dev)  # the last frame's radiance (relMSE)
    # warm-up: the first frames of the sequence rendered once, then commits up
    # to the next multiple of 32, so that the timed frames follow the
    # reference's schedule from frame 0 (runtime.hpp:124-125: a build whenever
    # geometry_updates % 32 == 0): build, 31 refits, build, refit
    backend.reset_history()
    for f in range(32):
        backend.model_update(ids[seq.CLOTH], cloth[f % seq.frames])
        backend.instances_commit(recs[f % seq.frames], rebuild_every=32)
        if f < 2:
            backend.render_resident_async(cams[f], cfg, 12345 + f, d_rgb.data_ptr())
    backend.sync()
    backend.reset_history()
    backend.stats_reset()
    backend.profile(1)
    st0 = backend.stats()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for f in range(seq.frames):
        backend.model_update(ids[seq.CLOTH], cloth[f])
        backend.instances_commit(recs[f], rebuild_every=32)
        last = f == seq.frames - 1
        backend.render_resident_async(cams[f], cfg, 12345 + f, d_rgb.data_ptr(), d_hdr.data_ptr() if last else None)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    secs = e0.elapsed_time(e1) / 1e3
    st = backend.stats()
    t = backend.stage_times()
    backend.profile(0)
    samples = st["path_samples"]
    render_ms = sum(v[0] for k, v in t.items() if k not in ("prep", "batch", "adjoint"))
    relmse = None
    g = ROOT / "tests" / "golden" / "relmse_sequence33.npz"
    if g.exists() and seq.frames == 34:
        ref = np.load(g)
        img = d_hdr.cpu().numpy().reshape(-1, 3)[ref["pixels"]].astype(np.float64)
        relmse = dict(frame=33, pixels=int(len(ref["pixels"])), ref_spp=int(ref["spp"]), spp=cfg.spp,
                      denoised=_relmse(img, ref["ref"]))
    return dict(workload=f"animated sequence: {seq.frames} frames at {seq.fps} fps, {cfg.width}x{cfg.height}, "
                         f"{cfg.spp} spp, depth {cfg.max_bounces}, {seq.n_tris:,} triangles ({len(seq.moving)} moving "
                         f"spheres, {len(cloth[0]):,}-triangle cloth), camera orbit {seq.orbit_deg} deg/frame, temporal "
                         "ReSTIR + denoise on animated geometry",
                value=samples / secs, unit="path samples/s", frames=seq.frames, ms_per_frame=1e3 * secs / seq.frames,
                wall_ms_per_frame=1e3 * wall / seq.frames, prep_ms_per_frame=t["prep"][0] / seq.frames,
                render_ms_per_frame=render_ms / seq.frames, bvh_builds=st["bvh_builds"] - st0["bvh_builds"],
                bvh_refits=st["bvh_refits"] - st0["bvh_refits"], h2d_bytes_per_frame=int(cloth[0].nbytes + recs[0].nbytes),
                path_samples=int(samples), relmse=relmse)


def _relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 0.01)))


def relmse_measure(backend, torch, cam, cfg, dev, seed):
    """relMSE of single frames against the FP64 16,384-spp references of
    tests/golden (make_relmse_refs.py: 4096 seeded pixels, the oracle's plain
    path tracer, same depth and clamp).  The CUDA frames are bit-identical to
    the oracle's fp32 frames on the same streams (the parity tests), so the CPU
    arm's relMSE at equal spp is the same.  For the headline workload: the
    denoised output and the raw ReSTIR radiance (denoiser off), each from a
    fresh history; for the Cornell box, its plain 16-spp frame (through
    rmcuda_render, which replaces the resident scene, so this runs last)."""
    from raymotion_b200.scene import RenderConfig  # noqa: F401  (cfg's type)
    from raymotion_b200.scenes import cornell_box
    golden = Path(__file__).resolve().parent / "tests" / "golden"
    out = {}
    g = golden / "relmse_icosphere720.npz"
    if g.exists():
        ref = np.load(g)
        pix, r = ref["pixels"], ref["ref"]
        npix = cfg.width * cfg.height
        d_rgb = torch.empty(npix * 3, dtype=torch.uint8, device=dev)
        d_hdr = torch.empty(npix * 3, dtype=torch.float32, device=dev)
        e = {}
        A = rb_abi()
        # switches from the flag bits (RM_FLAG_NO_ENV): the denoiser on, then off
        for name, flags in (("denoised", cfg.flags | A.RM_FLAG_NO_ENV),
                            ("restir_raw", cfg.flags | A.RM_FLAG_NO_ENV | A.RM_FLAG_DENOISE_OFF)):
            backend.reset_history()
            backend.render_resident_async(cam, dataclasses.replace(cfg, flags=flags), seed, d_rgb.data_ptr(),
                                          d_hdr.data_ptr())
            backend.sync()
            img = d_hdr.cpu().numpy().reshape(-1, 3)[pix].astype(np.float64)
            e[name] = _relmse(img, r)
        out["icosphere720"] = dict(pixels=int(len(pix)), ref_spp=int(ref["spp"]), spp=cfg.spp, **e)
    g = golden / "relmse_cornell.npz"
    if g.exists():
        ref = np.load(g)
        sb, ccam, ccfg = cornell_box(0)
        _, hdr = backend.render(sb.pack(), ccam, ccfg, seed, hdr=True, use_nodes=False)
        img = hdr.reshape(-1, 3)[ref["pixels"]].astype(np.float64)
        out["cornell"] = dict(pixels=int(len(ref["pixels"])), ref_spp=int(ref["spp"]), spp=ccfg.spp,
                              plain=_relmse(img, ref["ref"]))
    return out or None


def rb_abi():
    from raymotion_b200 import _abi
    return _abi


def screen_space_large(backend, torch, cam, cfg, dev, seed0, peak):
    """The screen-space passes where their working set exceeds L2.

    2048x1280 is the largest 16:10 frame whose ReSTIR buffers stay within the
    reference's 512 MiB limit (76 + 2 x 60 B per pixel, metal.mm:236-237); past
    it the reference drops ReSTIR and the denoiser.  1 spp keeps the frame
    cheap: the passes' work does not depend on spp.  Two frames build the
    temporal history, then five are timed per stage (events on the rendering
    stream): temporal 92 B/px, two a-trous passes 64 B/px each, tonemap write
    3 B/px, 223 B/px in all (585 MB per frame, above the 126 MB L2).
    """
    big = dataclasses.replace(cfg, width=2048, height=1280, spp=1)
    npix = big.width * big.height
    d_rgb = torch.empty(npix * 3, dtype=torch.uint8, device=dev)
    for i in range(2):
        backend.render_resident_async(cam, big, seed0 + i, d_rgb.data_ptr())
    backend.sync()
    backend.stats_reset()
    backend.profile(1)
    frames = 5
    for i in range(frames):
        backend.render_resident_async(cam, big, seed0 + 2 + i, d_rgb.data_ptr())
    backend.sync()
    t = backend.stage_times()
    backend.profile(0)
    ms = sum(t[k][0] for k in ("temporal", "atrous0", "atrous1")) / frames
    if ms <= 0:
        return None
    nbytes = npix * (92 + 64 + 64 + 3)
    ach = nbytes / (ms / 1e3) / 1e9
    passes = {}
    for k, b in (("temporal", 92), ("atrous0", 64), ("atrous1", 67)):
        us = t[k][0] / frames * 1e3
        if us > 0:
            passes[k] = dict(us=us, bytes_per_px=b, gbs=npix * b / us / 1e3, frac=npix * b / us / 1e3 / peak["hbm_gbs"])
    return dict(bound="hbm", kernels="k_denoise_temporal_tiled + k_denoise_atrous_tiled x2", width=big.width,
                height=big.height, achieved=ach, peak=peak["hbm_gbs"], unit="GB/s", frac=ach / peak["hbm_gbs"],
                us_per_frame=ms * 1e3, bytes_per_frame=nbytes, peak_source=peak["source"], passes=passes)


def run_b200(args, world, rank, local):
    import torch

    import raymotion_b200 as rb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene, cam, cfg, desc = workload(args.workload)
    backend = rb.Backend(local)
    # a dedicated stream: the rendering and the CUDA events that time it share it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    backend.set_stream(stream.cuda_stream)
    npix = cfg.width * cfg.height
    seed0 = 12345 + 1000 * rank
    # ---- device-resident frames (value)
    backend.upload(scene, use_nodes=False)
    if args.screen_space_only:
        print(json.dumps(screen_space_large(backend, torch, cam, cfg, dev, seed0 + 300, measured_peaks())), flush=True)
        backend.close()
        return 0
    d_rgb = torch.empty(npix * 3, dtype=torch.uint8, device=dev)
    for i in range(args.warmup):
        backend.render_resident_async(cam, cfg, seed0 + i, d_rgb.data_ptr())
    backend.sync()
    backend.stats_reset()
    backend.profile(1)
    torch.cuda.synchronize()
    barrier(world)
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        uuid = None
    clocks = Clocks(uuid)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.steps):
        backend.render_resident_async(cam, cfg, seed0 + args.warmup + k, d_rgb.data_ptr())
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    backend.sync()
    secs = ev0.elapsed_time(ev1) / 1e3
    st = backend.stats()
    wlog = backend.wave_log()  # of the last timed frame (the breakdown frame below runs with per-launch events)
    stage_t = backend.stage_times()
    stage_c = backend.stage_counters()
    secs_max, = allreduce([secs], "max", world, dev)
    samples_sum, rays_sum = allreduce([float(st["path_samples"]), float(st["rays"])], "sum", world, dev)
    value = samples_sum / secs_max
    # ---- per-kernel breakdown on one more (untimed) frame: every launch
    # event-timed, with the wavefront as one part so that launches do not
    # overlap (the timed frames run its parts on several streams)
    backend.stats_reset()
    backend.profile(2)
    parts_env = os.environ.get("RAYMOTION_CUDA_STREAMS")
    os.environ["RAYMOTION_CUDA_STREAMS"] = "1"
    if not args.no_breakdown:
        backend.render_resident_async(cam, cfg, seed0 + args.warmup + args.steps, d_rgb.data_ptr())
    backend.sync()
    if parts_env is None:
        del os.environ["RAYMOTION_CUDA_STREAMS"]
    else:
        os.environ["RAYMOTION_CUDA_STREAMS"] = parts_env
    kern_t = backend.stage_times()
    kern_c = backend.stage_counters()
    kern_st = backend.stats()
    backend.profile(0)
    wave_summary = None
    if len(wlog):
        act, us = wlog[:, 0], wlog[:, 3]
        first = int(act[0])
        marks = {}
        for f in (0.5, 0.1, 0.01):
            b = int(np.argmax(act < f * first))
            marks[f"batches_until_{int(f * 100)}pct"] = b
            marks[f"ms_until_{int(f * 100)}pct"] = float(us[b]) / 1e3
        wave_summary = dict(batches=int(len(act)), waves_per_batch=4, first_act=first, ms_loop=float(us[-1]) / 1e3,
                            **marks)
    # ---- roofline of the dominant kernel (the wavefront loop counts as its kernels)
    if args.no_breakdown:
        kern_t, kern_c = stage_t, stage_c
    kernel_stages = {k: v for k, v in kern_t.items() if k != "shade" or kern_t["wf_extend"][1] == 0}
    dom = max(kernel_stages, key=lambda k: kernel_stages[k][0])
    ms_total, launches = kern_t[dom]
    c = kern_c[dom]
    # one launch per wave traverses extension and shadow rays (k_wf_trace2):
    # its time is the extension stage's, its shadow rays' counters sit apart
    merged_trace = kern_t["wf_extend"][1] > 0 and kern_t["wf_shadow"][1] == 0
    if dom == "wf_extend" and merged_trace:
        c = {k: kern_c["wf_extend"][k] + kern_c["wf_shadow"][k] for k in c}
    if dom == "shade" and not c["nodes_visited"] and kern_c["wf_extend"]["nodes_visited"]:
        # without the per-launch breakdown the wavefront loop is timed as one
        # stage; its traversal counters sit with its traversal kernels
        c = {k: kern_c["wf_extend"][k] + kern_c["wf_shadow"][k] for k in c}
        dom = "wavefront shading loop"
    node_bytes = st.get("bvh_node_bytes", 64) or 64
    alg_bytes = (c["nodes_visited"] * node_bytes + c["tris_tested"] * 48) / max(launches, 1)
    avg_s = ms_total / 1e3 / max(launches, 1)
    peak = measured_peaks()
    achieved = alg_bytes / avg_s / 1e9 if avg_s > 0 else 0.0
    kernel_names = dict(plain="k_render_paths", shade="k_restir_shade", generate="k_restir_generate",
                        spatial="k_restir_spatial", temporal="k_denoise_temporal", atrous0="k_denoise_atrous",
                        atrous1="k_denoise_atrous", hash="k_hash", tonemap="k_tonemap",
                        wf_extend="k_wf_trace2" if merged_trace else "k_wf_extend",
                        wf_shadow="k_wf_shadow", wf_shade="k_wf_shade", wf_tail="k_wf_tail",
                        **{"wavefront shading loop": "k_wf_init + k_wf_trace + k_wf_shade (one stage)"})
    roofline = dict(bound="hbm", kernel=kernel_names.get(dom, dom), achieved=achieved, peak=peak["hbm_gbs"],
                    unit="GB/s", frac=achieved / peak["hbm_gbs"], traffic=ncu_traffic(kernel_names.get(dom, dom)),
                    peak_source=peak["source"],
                    mrays_per_s=c["rays"] / (ms_total * 1e3) if ms_total > 0 else None,
                    limiter=("traversal: latency and divergence of incoherent rays, fed from L1/L2 (DRAM a few per "
                             "cent busy); the HBM fraction is the rate at which node and triangle records are "
                             "fetched" if c["nodes_visited"] else "hbm"),
                    note=f"achieved = ({node_bytes} B x BVH nodes fetched + 48 B x triangle tests) per launch / "
                         "average launch time; most of these bytes hit L1/L2")
    # screen-space passes (temporal 92 B/px, two a-trous 64 B/px each, fused tonemap write 3 B/px):
    # algorithmic bytes per frame against the measured HBM peak
    ss_ms = sum(kern_t[k][0] for k in ("temporal", "atrous0", "atrous1"))
    ss_bytes = cfg.width * cfg.height * (92 + 64 + 64 + 3)
    roofline_ss = None
    if ss_ms > 0:
        ach = ss_bytes / (ss_ms / 1e3) / 1e9
        roofline_ss = dict(bound="hbm", kernels="k_denoise_temporal_tiled + k_denoise_atrous_tiled x2", achieved=ach,
                           peak=peak["hbm_gbs"], unit="GB/s", frac=ach / peak["hbm_gbs"], us_per_frame=ss_ms * 1e3,
                           bytes_per_frame=ss_bytes)
    stage_summary = {k: dict(ms_per_frame=v[0] / args.steps, launches_per_frame=v[1] / args.steps)
                     for k, v in stage_t.items() if v[1]}
    kernel_summary = {}
    for k, v in kern_t.items():
        if not v[1]:
            continue
        e = dict(ms=v[0], launches=v[1])
        rc = kern_c.get(k, {})
        if rc.get("rays"):
            e.update(rays=rc["rays"], nodes_per_ray=rc["nodes_visited"] / rc["rays"],
                     tests_per_ray=rc["tris_tested"] / rc["rays"], mrays_per_s=rc["rays"] / (v[0] * 1e3))
        if k == "wf_extend" and merged_trace:
            # extension and shadow rays of one launch per wave
            rs = kern_c["wf_shadow"]
            e.update(kernel="k_wf_trace2 (extension + shadow rays)", shadow_rays=rs["rays"],
                     shadow_nodes_per_ray=rs["nodes_visited"] / max(rs["rays"], 1),
                     mrays_per_s_both=(rc["rays"] + rs["rays"]) / (v[0] * 1e3))
        kernel_summary[k] = e
    ss_large = None if args.no_large else screen_space_large(backend, torch, cam, cfg, dev, seed0 + 300, peak)
    # ---- end to end through rmcuda_render with host buffers
    e2e = None
    if not args.no_e2e:
        pinned = {}
        for key in ("tris", "light_tri", "light_cdf", "texels"):
            a = getattr(scene, key)
            t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).pin_memory()
            pinned[key] = t.numpy().view(a.dtype).reshape(a.shape)
        hscene = rb.PackedScene(tris=pinned["tris"], light_tri=pinned["light_tri"], light_cdf=pinned["light_cdf"],
                                light_total=scene.light_total, texels=pinned["texels"], verts64=scene.verts64)
        out_t = torch.empty(npix * 3, dtype=torch.uint8).pin_memory()
        out = out_t.numpy()
        backend.render(hscene, cam, cfg, seed0 + 500, use_nodes=False, out=out)  # warm-up
        backend.stats_reset()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.steps):
            backend.render(hscene, cam, cfg, seed0 + 501 + k, use_nodes=False, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
        esec, = allreduce([e0.elapsed_time(e1) / 1e3], "max", world, dev)
        es, = allreduce([float(backend.stats()["path_samples"])], "sum", world, dev)
        h2d = sum(pinned[k].nbytes for k in pinned)
        e2e = dict(value=es / esec, unit=UNIT, h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(npix * 3),
                   ms_per_step=1e3 * esec / args.steps)
    # ---- relMSE against the FP64 references (before the steps that replace the resident scene)
    relmse = None if args.no_relmse else relmse_measure(backend, torch, cam, cfg, dev, seed0 + 900)
    # ---- batched vs serial rendering of many uneven scenes
    batch = None if args.no_batch else batch_compare(args, backend, torch, stream, dev, world)
    # ---- the animated sequence: device scene preparation + refit per frame
    sequence = None if args.no_sequence else sequence_measure(args, backend, torch, stream, dev)
    # ---- differentiable rendering: adjoint cost and a 200-step fit
    adjoint = None if args.no_adjoint else adjoint_measure(args, backend, torch, stream, dev, rank, world)
    # ---- CPU baseline (rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sample, threads, _, _ = cpu_band(scene, cam, cfg, args.cpu_seconds)
        cpu = dict(value=v, unit=UNIT, cores=threads, kind="port", sample=sample)
    if rank == 0:
        line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=1e3 * secs_max / args.steps, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="f32", data="synthetic (seeded procedural scene)",
                    config=dict(desc, parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
                    mrays_per_s=rays_sum / secs_max / 1e6, e2e=e2e, roofline=roofline, cpu_baseline=cpu,
                    kernel_attribution="kernels_one_frame and roofline: one more frame with every launch "
                                       "event-timed and the wavefront as one part (no overlapping launches); "
                                       "the timed frames run the wavefront's parts on their own streams",
                    gpu_launches=int(st["kernel_launches"]), clocks=clk, stages=stage_summary,
                    kernels_one_frame=kernel_summary, wavefront=wave_summary, roofline_screen_space=roofline_ss,
                    roofline_screen_space_large=ss_large,
                    batch=batch, adjoint=adjoint, sequence=sequence, relmse=relmse)
        print(json.dumps(line), flush=True)
    backend.close()
    return 0


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        return launch_ranks(args, sys.argv[1:])
    if int(os.environ.get("WORLD_SIZE", "1")) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={os.environ.get('WORLD_SIZE')} ranks were started",
              file=sys.stderr)
        return 2
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
