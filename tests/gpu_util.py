"""Helpers of the GPU parity tests."""
import numpy as np


def rel_close_fraction(a, b, rel=1e-4, abs_floor=1e-6):
    """Fraction of pixels whose three channels all satisfy |a-b| <= rel*|b| (+abs floor)."""
    a = np.asarray(a, np.float64).reshape(-1, 3)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    ok = np.abs(a - b) <= rel * np.abs(b) + abs_floor
    return ok.all(axis=1).mean()


def exact_fraction(a, b):
    a = np.asarray(a).reshape(-1, 3)
    b = np.asarray(b).reshape(-1, 3)
    return (a.view(np.uint32) == b.view(np.uint32)).all(axis=1).mean() if a.dtype == np.float32 else \
        (a == b).all(axis=1).mean()


def camera_rays(cam, cfg, jitter_seed=0):
    """Primary rays of render_paths (pathtrace.metal:729-737) with random jitter, 7 floats each."""
    rng = np.random.default_rng(jitter_seed)
    W, H = cfg.width, cfg.height
    y, x = np.mgrid[0:H, 0:W]
    sx = (x + rng.uniform(0, 1, x.shape) - W * 0.5).astype(np.float32).ravel()
    sy = (H * 0.5 - (y + rng.uniform(0, 1, y.shape))).astype(np.float32).ravel()
    f = np.float32(cam.focal)
    d = np.float32(1) / np.sqrt(sx * sx + (sy * sy + f * f))
    tx, ty, tz = sx * d, sy * d, f * d
    m = np.asarray(cam.m, np.float32)
    dx = tx * m[0] + (ty * m[1] + tz * m[2])
    dy = tx * m[3] + (ty * m[4] + tz * m[5])
    dz = tx * m[6] + (ty * m[7] + tz * m[8])
    n = len(sx)
    rays = np.zeros((n, 7), np.float32)
    rays[:, 0], rays[:, 1], rays[:, 2] = cam.x, cam.y, cam.z
    rays[:, 3], rays[:, 4], rays[:, 5] = dx, dy, dz
    rays[:, 6] = 1e30
    return rays


def random_rays(n, lo, hi, seed, tmax=1e30):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # a few axis-aligned directions exercise the 1e-30 guard of the slab test
    d[: n // 50] = np.eye(3)[rng.integers(0, 3, n // 50)] * rng.choice([-1, 1], (n // 50, 1))
    rays = np.zeros((n, 7), np.float32)
    rays[:, :3] = o
    rays[:, 3:6] = d
    rays[:, 6] = tmax
    return rays
