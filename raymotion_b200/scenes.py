"""Seeded synthetic scenes of the benchmark workloads (no external assets).

* ``cornell_box(seed)``: 36 triangles - five walls (albedo 0.75 grey, left
  wall red 0.63/0.065/0.05, right wall green 0.14/0.45/0.09), a tall diffuse
  box, a short GGX-metal box of roughness 0.3 and one emissive quad light of
  radiance (17, 12, 4); box placement and the camera are drawn from ``seed``.
* ``icosphere_field(...)``: instanced icospheres (subdivision 4, 5120
  triangles each) displaced by seeded 3-D value noise of amplitude 0.05 r,
  radii uniform in [0.2, 1.5], centres uniform in a 40 x 10 x 40 box, a ground
  plane, materials 50 % diffuse (albedo U[0.1, 0.9]^3) / 30 % GGX metal
  (roughness U[0.05, 1]) / 20 % dielectric (IOR 1.5, roughness 0 or 0.2), and
  small emissive triangles with log-uniform radiance in [1, 100].  The default
  arguments give 200 spheres + 2 + 4096 = 1,028,098 triangles.
* ``batch_workload(...)``: many such scenes of uneven size for batched
  rendering: triangle counts log-uniform over [1k, 2M], resolutions from
  {256x256, 640x360, 1280x720, 1920x1080}, spp from {4, 16, 64}, depth 8-12,
  all on the plain path (ReSTIR and the denoiser off).
* ``AnimatedSequence(...)``: the icosphere field as models and instances
  (one object-space model per sphere), 20 % of the spheres moving rigidly
  along seeded sinusoids, a 256 x 256-vertex cloth (130,050 triangles)
  deformed by seeded sine waves, and a camera orbiting 6 degrees per frame;
  34 frames at 30 fps, 1280x720, 16 spp, temporal ReSTIR and denoise on the
  animated geometry.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi
from .scene import Camera, RenderConfig, SceneBuilder


def _quad(sb: SceneBuilder, a, b, c, d, normal=None, **mat) -> None:
    a, b, c, d = (np.asarray(x, np.float64) for x in (a, b, c, d))
    n = None if normal is None else [normal]
    sb.add_triangles([a], [b], [c], n, n, n, **mat)
    sb.add_triangles([a], [c], [d], n, n, n, **mat)


def _box(sb: SceneBuilder, center, half, angle_deg, **mat) -> None:
    cx, cy, cz = center
    hx, hy, hz = half
    ca, sa = math.cos(math.radians(angle_deg)), math.sin(math.radians(angle_deg))

    def p(x, y, z):
        return (cx + ca * x - sa * z, cy + y, cz + sa * x + ca * z)

    corners = {(i, j, k): p(i * hx, j * hy, k * hz) for i in (-1, 1) for j in (-1, 1) for k in (-1, 1)}
    faces = [  # (corner keys counter-clockwise seen from outside), outward normal in box space
        ([(-1, 1, -1), (-1, 1, 1), (1, 1, 1), (1, 1, -1)], (0, 1, 0)),
        ([(-1, -1, -1), (1, -1, -1), (1, -1, 1), (-1, -1, 1)], (0, -1, 0)),
        ([(-1, -1, -1), (-1, 1, -1), (1, 1, -1), (1, -1, -1)], (0, 0, -1)),
        ([(-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)], (0, 0, 1)),
        ([(-1, -1, -1), (-1, -1, 1), (-1, 1, 1), (-1, 1, -1)], (-1, 0, 0)),
        ([(1, -1, -1), (1, 1, -1), (1, 1, 1), (1, -1, 1)], (1, 0, 0)),
    ]
    for keys, (nx, ny, nz) in faces:
        n = (ca * nx - sa * nz, ny, sa * nx + ca * nz)
        _quad(sb, *(corners[k] for k in keys), normal=n, **mat)


def cornell_box(seed: int = 0):
    """Returns (SceneBuilder, Camera, RenderConfig) of the 320x180 / 16 spp / depth 8 workload."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    grey, red, green = (0.75, 0.75, 0.75), (0.63, 0.065, 0.05), (0.14, 0.45, 0.09)
    _quad(sb, (-1, 0, 0), (1, 0, 0), (1, 0, 2), (-1, 0, 2), normal=(0, 1, 0), albedo=grey)     # floor
    _quad(sb, (-1, 2, 0), (-1, 2, 2), (1, 2, 2), (1, 2, 0), normal=(0, -1, 0), albedo=grey)    # ceiling
    _quad(sb, (-1, 0, 2), (1, 0, 2), (1, 2, 2), (-1, 2, 2), normal=(0, 0, -1), albedo=grey)    # back
    _quad(sb, (-1, 0, 0), (-1, 0, 2), (-1, 2, 2), (-1, 2, 0), normal=(1, 0, 0), albedo=red)    # left
    _quad(sb, (1, 0, 0), (1, 2, 0), (1, 2, 2), (1, 0, 2), normal=(-1, 0, 0), albedo=green)     # right
    j = rng.uniform(-0.08, 0.08, size=4)
    _box(sb, (-0.35 + j[0], 0.6, 1.3 + j[1]), (0.28, 0.6, 0.28), 17 + 10 * j[2], albedo=grey)
    _box(sb, (0.38 + j[3], 0.3, 0.7), (0.27, 0.3, 0.27), -18, albedo=(0.8, 0.8, 0.8), metallic=1.0, rough=0.3)
    # emitters are one-sided along their geometric normal (v1-v0)x(v2-v0): wind it downwards
    _quad(sb, (-0.25, 1.98, 0.75), (0.25, 1.98, 0.75), (0.25, 1.98, 1.25), (-0.25, 1.98, 1.25),
          normal=(0, -1, 0), albedo=(0.78, 0.78, 0.78), emission=(17, 12, 4))
    cj = rng.uniform(-0.05, 0.05, size=3)
    cam = Camera().set((cj[0], 1.0 + cj[1], -2.2 + cj[2]), (0, 0, 0), 106)
    # config 0 as stated: NEE + MIS, Russian roulette off (the reference always applies it; RM_FLAG_NO_RR)
    cfg = RenderConfig(width=320, height=180, spp=16, max_bounces=8, restir_candidates=1, restir_spatial=0,
                       flags=_abi.RM_FLAG_NO_RR)
    return sb, cam, cfg


def _icosphere(subdiv: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.asarray(v), np.asarray(faces, np.int64)


def _value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise in [-1, 1] on the integer lattice, hashed from ``seed``."""
    base = np.floor(p).astype(np.int64)
    f = p - base
    w = f * f * (3 - 2 * f)

    def h(ix, iy, iz):
        z = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        z = (z ^ (z >> 13)) * 1274126177
        z = z ^ (z >> 16)
        return ((z & 0xFFFF) / 32767.5) - 1.0

    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out = out + wx * wy * wz * h(base[:, 0] + dx, base[:, 1] + dy, base[:, 2] + dz)
    return out


def _displaced_sphere(unit_v, faces, center, r, noise_seed):
    """Corners and smooth vertex normals of an icosphere of radius r displaced by
    value noise of amplitude 0.05 r."""
    world = center + unit_v * r
    disp = 0.05 * r * _value_noise(world * (2.0 / r), noise_seed)
    pos = center + unit_v * (r + disp)[:, None]
    fa, fb, fc = pos[faces[:, 0]], pos[faces[:, 1]], pos[faces[:, 2]]
    fn = np.cross(fb - fa, fc - fa)
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, faces[:, k], fn)
    vn /= np.linalg.norm(vn, axis=1, keepdims=True)
    return fa, fb, fc, vn[faces[:, 0]], vn[faces[:, 1]], vn[faces[:, 2]]


def icosphere_field(seed: int = 1, n_spheres: int = 200, subdiv: int = 4, n_emitters: int = 4096,
                    width: int = 1280, height: int = 720, spp: int = 64, depth: int = 12):
    """Returns (SceneBuilder, Camera, RenderConfig) of the instanced icosphere workload."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    unit_v, faces = _icosphere(subdiv)
    radii = rng.uniform(0.2, 1.5, n_spheres)
    centers = np.stack([rng.uniform(-20, 20, n_spheres), rng.uniform(0, 10, n_spheres),
                        rng.uniform(-20, 20, n_spheres)], axis=1)
    kind = rng.choice(3, size=n_spheres, p=[0.5, 0.3, 0.2])
    for i in range(n_spheres):
        fa, fb, fc, na, nb, nc = _displaced_sphere(unit_v, faces, centers[i], radii[i], seed * 1000 + i)
        if kind[i] == 0:
            mat = dict(albedo=tuple(rng.uniform(0.1, 0.9, 3)), rough=0.5)
        elif kind[i] == 1:
            mat = dict(albedo=tuple(rng.uniform(0.5, 0.95, 3)), metallic=1.0, rough=float(rng.uniform(0.05, 1.0)))
        else:
            mat = dict(albedo=(1.0, 1.0, 1.0), ior=1.5, rough=float(rng.choice([0.0, 0.2])))
        sb.add_triangles(fa, fb, fc, na, nb, nc, **mat)
    g = 100.0
    _quad(sb, (-g, 0, -g), (-g, 0, g), (g, 0, g), (g, 0, -g), normal=(0, 1, 0), albedo=(0.5, 0.5, 0.5), rough=0.8)
    # small emitters facing down, scattered above the spheres
    c = np.stack([rng.uniform(-24, 24, n_emitters), rng.uniform(11, 14, n_emitters),
                  rng.uniform(-24, 24, n_emitters)], axis=1)
    s = rng.uniform(0.15, 0.35, n_emitters)[:, None]
    a0 = c + np.concatenate([-s, 0 * s, -s], axis=1)
    a1 = c + np.concatenate([s, 0 * s, -s * 0.2], axis=1)
    a2 = c + np.concatenate([-s * 0.3, 0 * s, s], axis=1)
    radiance = np.exp(rng.uniform(math.log(1.0), math.log(100.0), n_emitters))
    tint = rng.uniform(0.6, 1.0, (n_emitters, 3))
    down = np.broadcast_to(np.asarray([0.0, -1.0, 0.0]), (n_emitters, 3))
    sb.add_triangles(a0, a1, a2, down, down, down, albedo=(0.8, 0.8, 0.8), emission=tint * radiance[:, None])
    cam = Camera().set((0.0, 9.0, -34.0), (14.0, 0.0, 0.0), 60)
    cfg = RenderConfig(width=width, height=height, spp=spp, max_bounces=depth, restir_candidates=32,
                       restir_spatial=5, restir_radius=30.0)
    return sb, cam, cfg


PLAIN_FLAGS = _abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_RESTIR_OFF | _abi.RM_FLAG_DENOISE_OFF
BATCH_RESOLUTIONS = ((256, 256), (640, 360), (1280, 720), (1920, 1080))


def sized_field(seed: int, n_tris: int, width: int, height: int, spp: int, depth: int):
    """An icosphere field of about ``n_tris`` triangles on the plain path.

    Emitters: n_tris / 64 clamped to [16, 4096]; the rest are icospheres of the
    finest subdivision (<= 4) that still gives at least three spheres, plus the
    two ground triangles."""
    n_emit = int(min(4096, max(16, n_tris // 64)))
    rest = max(20, n_tris - n_emit - 2)
    subdiv = 0
    for k in (4, 3, 2, 1, 0):
        if rest // (20 * 4 ** k) >= 3:
            subdiv = k
            break
    n_spheres = max(1, int(round(rest / (20 * 4 ** subdiv))))
    sb, cam, cfg = icosphere_field(seed, n_spheres=n_spheres, subdiv=subdiv, n_emitters=n_emit, width=width,
                                   height=height, spp=spp, depth=depth)
    cfg.flags = PLAIN_FLAGS
    return sb, cam, cfg


def batch_workload(seed: int = 3, n_scenes: int = 64, tri_range=(1000, 2_000_000), resolutions=BATCH_RESOLUTIONS,
                   spps=(4, 16, 64), depths=(8, 12)):
    """Specs of a batch of uneven scenes: a list of dicts (seed, n_tris, width,
    height, spp, depth) drawn from ``seed``; ``sized_field(**spec)`` builds one."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = math.log(tri_range[0]), math.log(tri_range[1])
    for i in range(n_scenes):
        n_tris = int(round(math.exp(rng.uniform(lo, hi))))
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        spp = int(spps[int(rng.integers(len(spps)))])
        depth = int(rng.integers(depths[0], depths[1] + 1))
        out.append(dict(seed=seed * 1000 + i, n_tris=n_tris, width=w, height=h, spp=spp, depth=depth))
    return out


# parameter ranges of the inverse-rendering materials (albedo rgb, rough, emission rgb, ior)
INVERSE_LO = np.array([0.05, 0.05, 0.05, 0.05, 0.0, 0.0, 0.0, 1.3], np.float32)
INVERSE_HI = np.array([0.95, 0.95, 0.95, 1.0, 20.0, 20.0, 20.0, 1.7], np.float32)


def inverse_scene(seed: int = 4, n_spheres: int = 100, subdiv: int = 3, ground: int = 190, patches=(10, 14),
                  n_emitters: int = 16, n_dielectric: int = 32, width: int = 512, height: int = 512, spp: int = 32,
                  depth: int = 8):
    """The differentiable-rendering scene: displaced icospheres (20 * 4**subdiv
    triangles each) over a tessellated ground of ground x ground quads split
    into patches[0] x patches[1] material patches, and n_emitters small quad
    lights.  Materials: one per sphere, per ground patch and per light
    (100 + 140 + 16 = 256 by default), parameters uniform in INVERSE_LO..HI
    (emission only for the lights, ior only for n_dielectric spheres; the
    others keep emission 0 and ior 1).  The defaults give 100 * 1280 + 72,200 +
    32 = 200,232 triangles.  Returns a dict: scene (PackedScene with the
    materials applied), tri_material, params (n x 8 float32), mask (n x 8 bool,
    the parameters a fit may change), camera, config (plain path, fixed spp)."""
    rng = np.random.default_rng(seed)
    sb = SceneBuilder()
    unit_v, faces = _icosphere(subdiv)
    n_patch = patches[0] * patches[1]
    n_mat = n_spheres + n_patch + n_emitters
    params = np.zeros((n_mat, 8), np.float32)
    params[:, 0:3] = rng.uniform(INVERSE_LO[0], INVERSE_HI[0], (n_mat, 3))
    params[:, 3] = rng.uniform(INVERSE_LO[3], INVERSE_HI[3], n_mat)
    params[:, 7] = 1.0
    mask = np.zeros((n_mat, 8), bool)
    mask[:, 0:4] = True
    diel = rng.choice(n_spheres, size=min(n_dielectric, n_spheres), replace=False)
    params[diel, 7] = rng.uniform(INVERSE_LO[7], INVERSE_HI[7], len(diel))
    mask[diel, 7] = True
    lights = np.arange(n_spheres + n_patch, n_mat)
    params[lights, 4:7] = rng.uniform(INVERSE_LO[4], INVERSE_HI[4], (len(lights), 3))
    mask[lights, 4:7] = True
    metal = rng.uniform(size=n_spheres) < 0.3
    tri_mat = []
    radii = rng.uniform(0.5, 1.5, n_spheres)
    centers = np.stack([rng.uniform(-12, 12, n_spheres), rng.uniform(0.5, 4, n_spheres),
                        rng.uniform(-12, 12, n_spheres)], axis=1)
    for i in range(n_spheres):
        fa, fb, fc, na, nb, nc = _displaced_sphere(unit_v, faces, centers[i], radii[i], seed * 1000 + i)
        is_diel = params[i, 7] > 1.0001
        idx = sb.add_triangles(fa, fb, fc, na, nb, nc, albedo=tuple(params[i, 0:3]), rough=float(params[i, 3]),
                               metallic=1.0 if (metal[i] and not is_diel) else 0.0, ior=float(params[i, 7]))
        tri_mat.append(np.full(len(idx), i, np.int32))
    g = 20.0
    xs = np.linspace(-g, g, ground + 1)
    ix, iz = np.meshgrid(np.arange(ground), np.arange(ground), indexing="ij")
    ix, iz = ix.ravel(), iz.ravel()
    y0 = np.zeros(len(ix))
    a = np.stack([xs[ix], y0, xs[iz]], axis=1)
    b = np.stack([xs[ix], y0, xs[iz + 1]], axis=1)
    c = np.stack([xs[ix + 1], y0, xs[iz + 1]], axis=1)
    d = np.stack([xs[ix + 1], y0, xs[iz]], axis=1)
    pm = n_spheres + (ix * patches[0] // ground) * patches[1] + (iz * patches[1] // ground)
    up = np.broadcast_to(np.asarray([0.0, 1.0, 0.0]), (len(ix), 3))
    for tri in ((a, b, c), (a, c, d)):
        sb.add_triangles(tri[0], tri[1], tri[2], up, up, up, albedo=params[pm, 0:3], rough=params[pm, 3])
        tri_mat.append(pm.astype(np.int32))
    lc = np.stack([rng.uniform(-10, 10, n_emitters), rng.uniform(8, 11, n_emitters),
                   rng.uniform(-10, 10, n_emitters)], axis=1)
    h = 0.6
    down = np.broadcast_to(np.asarray([0.0, -1.0, 0.0]), (n_emitters, 3))
    p0 = lc + [-h, 0, -h]
    p1 = lc + [h, 0, -h]
    p2 = lc + [h, 0, h]
    p3 = lc + [-h, 0, h]
    for tri in ((p0, p1, p2), (p0, p2, p3)):
        sb.add_triangles(tri[0], tri[1], tri[2], down, down, down, albedo=params[lights, 0:3],
                         rough=params[lights, 3], emission=params[lights, 4:7])
        tri_mat.append(lights.astype(np.int32))
    tri_mat = np.concatenate(tri_mat)
    packed = sb.pack()
    assert len(tri_mat) == packed.n_tris
    from .scene import with_materials
    packed = with_materials(packed, tri_mat, params)
    cam = Camera().set((0.0, 12.0, -27.0), (22.0, 0.0, 0.0), 58)
    cfg = RenderConfig(width=width, height=height, spp=spp, max_bounces=depth, adapt_min=0, restir_candidates=1,
                       restir_spatial=0, flags=PLAIN_FLAGS | _abi.RM_FLAG_NOADAPT)
    return dict(scene=packed, tri_material=tri_mat, params=params, mask=mask, camera=cam, config=cfg)


class AnimatedSequence:
    """The animated sequence: models, per-frame instances, cloth and camera.

    ``models`` lists object-space triangle arrays (``_abi.MODEL_TRI_DTYPE``):
    the 200 spheres (each displaced by its own noise, centred on the origin),
    the ground, the 4096 emitters and the cloth at frame 0 (``CLOTH`` is its
    index).  ``instances(f)`` places them at frame ``f`` (time f / fps);
    ``cloth(f)`` is the cloth model at frame ``f``; ``camera(f)`` orbits the
    field centre by ``orbit_deg`` per frame.
    """

    def __init__(self, seed: int = 1, n_spheres: int = 200, subdiv: int = 4, n_emitters: int = 4096,
                 cloth_verts: int = 256, frames: int = 34, fps: int = 30, orbit_deg: float = 6.0,
                 width: int = 1280, height: int = 720, spp: int = 16, depth: int = 12, moving: float = 0.2):
        from .objects import Instance, model_from_arrays
        self._Instance = Instance
        self._model = model_from_arrays
        rng = np.random.default_rng(seed)
        self.frames, self.fps, self.orbit_deg = frames, fps, orbit_deg
        unit_v, faces = _icosphere(subdiv)
        radii = rng.uniform(0.2, 1.5, n_spheres)
        self.centers = np.stack([rng.uniform(-20, 20, n_spheres), rng.uniform(0, 10, n_spheres),
                                 rng.uniform(-20, 20, n_spheres)], axis=1)
        kind = rng.choice(3, size=n_spheres, p=[0.5, 0.3, 0.2])
        origin = np.zeros(3)
        self.models = []
        for i in range(n_spheres):
            fa, fb, fc, na, nb, nc = _displaced_sphere(unit_v, faces, origin, radii[i], seed * 1000 + i)
            if kind[i] == 0:
                mat = dict(albedo=tuple(rng.uniform(0.1, 0.9, 3)), rough=0.5)
            elif kind[i] == 1:
                mat = dict(albedo=tuple(rng.uniform(0.5, 0.95, 3)), metallic=1.0, rough=float(rng.uniform(0.05, 1.0)))
            else:
                mat = dict(albedo=(1.0, 1.0, 1.0), ior=1.5, rough=float(rng.choice([0.0, 0.2])))
            self.models.append(model_from_arrays(fa, fb, fc, na, nb, nc, **mat))
        g = 100.0
        up = np.array([0.0, 1.0, 0.0])
        self.models.append(model_from_arrays([[-g, 0, -g], [-g, 0, -g]], [[-g, 0, g], [g, 0, g]],
                                             [[g, 0, g], [g, 0, -g]], [up, up], [up, up], [up, up],
                                             albedo=(0.5, 0.5, 0.5), rough=0.8))
        c = np.stack([rng.uniform(-24, 24, n_emitters), rng.uniform(11, 14, n_emitters),
                      rng.uniform(-24, 24, n_emitters)], axis=1)
        s = rng.uniform(0.15, 0.35, n_emitters)[:, None]
        a0 = c + np.concatenate([-s, 0 * s, -s], axis=1)
        a1 = c + np.concatenate([s, 0 * s, -s * 0.2], axis=1)
        a2 = c + np.concatenate([-s * 0.3, 0 * s, s], axis=1)
        radiance = np.exp(rng.uniform(math.log(1.0), math.log(100.0), n_emitters))
        tint = rng.uniform(0.6, 1.0, (n_emitters, 3))
        down = np.broadcast_to(np.asarray([0.0, -1.0, 0.0]), (n_emitters, 3))
        self.models.append(model_from_arrays(a0, a1, a2, down, down, down, albedo=(0.8, 0.8, 0.8),
                                             emission=tint * radiance[:, None]))
        # moving spheres: a seeded sinusoid per axis
        self.moving = rng.choice(n_spheres, size=int(round(moving * n_spheres)), replace=False)
        nm = len(self.moving)
        self.amp = rng.uniform(0.5, 2.0, (nm, 3)) * np.array([1.0, 0.3, 1.0])
        self.omega = rng.uniform(1.0, 3.0, (nm, 3))
        self.phase = rng.uniform(0, 2 * math.pi, (nm, 3))
        # cloth: a curtain behind the field, waves across it
        self.cloth_n = cloth_verts
        u = np.linspace(-16.0, 16.0, cloth_verts)
        v = np.linspace(0.5, 12.5, cloth_verts)
        self._cu, self._cv = np.meshgrid(u, v, indexing="xy")
        k = rng.uniform(0.3, 0.8, 2)
        w = rng.uniform(1.0, 2.5, 2)
        ph = rng.uniform(0, 2 * math.pi, 2)
        self._wave = (k, w, ph)
        q = np.arange(cloth_verts - 1)
        i00 = (q[None, :] + cloth_verts * q[:, None]).ravel()
        self._tri = np.concatenate([np.stack([i00, i00 + 1, i00 + cloth_verts + 1], axis=1),
                                    np.stack([i00, i00 + cloth_verts + 1, i00 + cloth_verts], axis=1)])
        self.CLOTH = len(self.models)
        self.models.append(self.cloth(0))
        self.cfg = RenderConfig(width=width, height=height, spp=spp, max_bounces=depth, restir_candidates=32,
                                restir_spatial=5, restir_radius=30.0, flags=_abi.RM_FLAG_ANIMATED_HISTORY)

    def time(self, f: int) -> float:
        return f / self.fps

    def cloth(self, f: int) -> np.ndarray:
        t = self.time(f)
        (kx, ky), (wx, wy), (px, py) = self._wave
        x, y = self._cu, self._cv
        z = 24.0 + 0.8 * np.sin(kx * x + wx * t + px) + 0.5 * np.sin(ky * y + wy * t + py)
        dzdx = 0.8 * kx * np.cos(kx * x + wx * t + px)
        dzdy = 0.5 * ky * np.cos(ky * y + wy * t + py)
        pos = np.stack([x, y, z], axis=-1).reshape(-1, 3)
        nrm = np.stack([-dzdx, -dzdy, np.ones_like(z)], axis=-1).reshape(-1, 3)
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        tri = self._tri
        return self._model(pos[tri[:, 0]], pos[tri[:, 1]], pos[tri[:, 2]], nrm[tri[:, 0]], nrm[tri[:, 1]],
                           nrm[tri[:, 2]], albedo=(0.7, 0.15, 0.1), rough=0.7)

    def instances(self, f: int) -> list:
        t = self.time(f)
        pos = self.centers.copy()
        pos[self.moving] += self.amp * np.sin(self.omega * t + self.phase)
        out = [self._Instance(model=i, position=tuple(pos[i])) for i in range(len(self.centers))]
        out += [self._Instance(model=len(self.centers)), self._Instance(model=len(self.centers) + 1),
                self._Instance(model=self.CLOTH)]
        return out

    def camera(self, f: int) -> Camera:
        th = self.orbit_deg * f
        r = math.radians(th)
        return Camera().set((-34.0 * math.sin(r), 9.0, -34.0 * math.cos(r)), (14.0, th, 0.0), 60)

    @property
    def n_tris(self) -> int:
        return sum(len(m) for m in self.models)
