"""Caller-side scene model: what the reference engine hands to its backend.

The reference keeps scenes in fp64 (include/raymotion/scene.hpp:26-96); every
triangle is precomputed by Scene::add_triangle (src/engine/scene.cpp:16-87):
edge cross-product normal n, its normalisation nn, degenerate rejection
|d00*d11 - d01^2| <= 1e-12, axis-aligned bounds, alpha clamped to [0, 1], and
for emissive triangles a running CDF of area x luminance.  The camera is
Camera::update_trig / update_focal (src/engine/camera.cpp:3-22) and the render
settings are RenderConfig (include/raymotion/pathtrace.hpp:54-81).

``SceneBuilder`` is the same model, vectorised with numpy so that the
million-triangle synthetic scenes build in about a second; ``pack()`` yields
the fp32 buffers that the reference's Metal host code uploads
(src/engine/metal.mm:109-145) and that the C ABI of librmcuda takes.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi


def _cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    # component formulas of Vec3 cross (include/raymotion/math.hpp:50-56)
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def _dot(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]


def _normalize(v: np.ndarray) -> np.ndarray:
    l = np.sqrt(_dot(v, v))
    out = np.zeros_like(v)
    ok = ~(l < 1e-30)
    out[ok] = v[ok] / l[ok, None]
    return out


@dataclass
class Texture:
    width: int
    height: int
    pixels: np.ndarray  # (height*width, 3) linear RGB, top row first


@dataclass
class PackedScene:
    """fp32 buffers of one frame (the arguments of rmcuda_render)."""
    tris: np.ndarray                  # TRIANGLE_DTYPE
    light_tri: np.ndarray             # int32
    light_cdf: np.ndarray             # float32
    light_total: float
    texels: np.ndarray                # (n, 3) float32
    verts64: np.ndarray               # (n, 9) float64, for CPU BVH builders
    nodes: np.ndarray | None = None   # BVH_NODE_DTYPE, caller BVH (None: device build)
    bvh_tri: np.ndarray | None = None

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])

    def view(self, use_nodes: bool = True) -> _abi.RmSceneView:
        v = _abi.RmSceneView()
        v.tris = _abi.ptr(self.tris) if self.n_tris else None
        v.n_tris = self.n_tris
        if use_nodes and self.nodes is not None:
            v.nodes = _abi.ptr(self.nodes) if len(self.nodes) else C.cast(C.pointer(C.c_int(0)), C.c_void_p).value
            v.n_nodes = len(self.nodes)
            v.bvh_tri = _abi.ptr(self.bvh_tri) if self.bvh_tri is not None and len(self.bvh_tri) else None
        else:
            v.nodes = None
            v.n_nodes = 0
            v.bvh_tri = None
        v.light_tri = _abi.ptr(self.light_tri) if len(self.light_tri) else None
        v.light_cdf = _abi.ptr(self.light_cdf) if len(self.light_cdf) else None
        v.n_lights = len(self.light_tri)
        v.light_total = float(self.light_total)
        v.texels = _abi.ptr(self.texels) if len(self.texels) else None
        v.n_texels = len(self.texels)
        return v


MATERIAL_PARAMS = 8  # albedo rgb, rough, emission rgb, ior (rm_material)


def light_table(scene: PackedScene, emission: np.ndarray) -> tuple[np.ndarray, float]:
    """Light-selection CDF over scene.light_tri by area x luminance (scene.cpp:73-85)
    for per-triangle emission (n_tris x 3); returns (cdf float32, total)."""
    lt = scene.light_tri
    if not len(lt):
        return np.zeros(0, np.float32), 0.0
    v = scene.verts64[lt]
    e1 = v[:, 3:6] - v[:, 0:3]
    e2 = v[:, 6:9] - v[:, 0:3]
    d00 = np.einsum("ij,ij->i", e1, e1)
    d01 = np.einsum("ij,ij->i", e1, e2)
    d11 = np.einsum("ij,ij->i", e2, e2)
    area = 0.5 * np.sqrt(np.maximum(d00 * d11 - d01 * d01, 0.0))
    em = np.asarray(emission, np.float64)[lt]
    lum = np.maximum(0.2126 * em[:, 0] + 0.7152 * em[:, 1] + 0.0722 * em[:, 2], 1e-6)
    cdf = np.add.accumulate(area * lum)
    return cdf.astype(np.float32), float(np.float32(cdf[-1]))


def with_materials(scene: PackedScene, tri_material: np.ndarray, params: np.ndarray) -> PackedScene:
    """A copy of ``scene`` whose triangles take their material's albedo, rough,
    emission and ior (params: n_materials x 8 float32; tri_material -1 keeps a
    triangle's own values), with the light table recomputed from the new
    emission; the host-side twin of rmcuda_scene_set_materials."""
    tm = np.asarray(tri_material, np.int32)
    prm = np.asarray(params, np.float32)
    t = scene.tris.copy()
    sel = tm >= 0
    m = tm[sel]
    for k, name in enumerate(("ar", "ag", "ab", "rough", "er", "eg", "eb", "ior")):
        t[name][sel] = prm[m, k]
    emission = np.stack([t["er"], t["eg"], t["eb"]], axis=1).astype(np.float64)
    cdf, total = light_table(scene, emission)
    return PackedScene(tris=t, light_tri=scene.light_tri, light_cdf=cdf, light_total=np.float32(total),
                       texels=scene.texels, verts64=scene.verts64, nodes=scene.nodes, bvh_tri=scene.bvh_tri)


class SceneBuilder:
    """fp64 scene with the reference's add_triangle precompute, vectorised."""

    def __init__(self) -> None:
        self._chunks: list[dict[str, np.ndarray]] = []
        self.textures: list[Texture] = []

    def add_texture(self, tex: Texture) -> int:
        self.textures.append(tex)
        return len(self.textures) - 1

    def add_triangles(self, p0, p1, p2, n0=None, n1=None, n2=None, *, albedo=(1.0, 1.0, 1.0),
                      emission=(0.0, 0.0, 0.0), metallic=0.0, ior=1.0, rough=0.5, shader=0, alpha=1.0,
                      uv=None, texture: int = -1) -> np.ndarray:
        """Add triangles; per-triangle attributes broadcast.  Returns the new indices (-1 if rejected)."""
        p0 = np.atleast_2d(np.asarray(p0, np.float64))
        p1 = np.atleast_2d(np.asarray(p1, np.float64))
        p2 = np.atleast_2d(np.asarray(p2, np.float64))
        m = p0.shape[0]
        e1 = p1 - p0
        e2 = p2 - p0
        n = _cross(e1, e2)
        d00 = _dot(e1, e1)
        d01 = _dot(e1, e2)
        d11 = _dot(e2, e2)
        denom = d00 * d11 - d01 * d01
        keep = ~(np.abs(denom) <= 1e-12)
        if n0 is None:
            fn = _normalize(n)
            n0 = n1 = n2 = fn
        n0 = np.broadcast_to(np.asarray(n0, np.float64), (m, 3))
        n1 = np.broadcast_to(np.asarray(n1, np.float64), (m, 3))
        n2 = np.broadcast_to(np.asarray(n2, np.float64), (m, 3))

        def col(x, k=None):
            a = np.asarray(x, np.float64)
            if k is not None:
                return np.broadcast_to(a, (m, k)).astype(np.float64)
            return np.broadcast_to(a, (m,)).astype(np.float64)

        alb = col(albedo, 3)
        emi = col(emission, 3)
        al = col(alpha)
        al = np.where(np.isfinite(al), np.clip(al, 0.0, 1.0), 1.0)
        uvs = np.zeros((m, 6)) if uv is None else np.broadcast_to(np.asarray(uv, np.float64), (m, 6))
        chunk = dict(p0=p0[keep], p1=p1[keep], p2=p2[keep], n=n[keep], nn=_normalize(n[keep]),
                     n0=np.ascontiguousarray(n0[keep]), n1=np.ascontiguousarray(n1[keep]),
                     n2=np.ascontiguousarray(n2[keep]), alb=alb[keep], emi=emi[keep],
                     metallic=col(metallic)[keep], ior=col(ior)[keep], rough=col(rough)[keep],
                     shader=np.broadcast_to(np.asarray(shader, np.int32), (m,))[keep].copy(),
                     alpha=al[keep], uv=np.ascontiguousarray(uvs[keep]),
                     texture=np.broadcast_to(np.asarray(texture, np.int32), (m,))[keep].copy(),
                     area2=denom[keep])
        start = sum(len(c["p0"]) for c in self._chunks)
        self._chunks.append(chunk)
        idx = np.full(m, -1, np.int64)
        idx[keep] = start + np.arange(int(keep.sum()))
        return idx

    def add_triangle(self, p0, p1, p2, u0=0, v0=0, u1=0, v1=0, u2=0, v2=0, n0=None, n1=None, n2=None,
                     ar=1.0, ag=1.0, ab=1.0, er=0.0, eg=0.0, eb=0.0, metallic=0.0, ior=1.0, rough=0.5,
                     shader=0, alpha=1.0) -> int:
        """Scalar form with the argument order of Scene::add_triangle (scene.hpp:91-95)."""
        idx = self.add_triangles([p0], [p1], [p2], None if n0 is None else [n0], None if n1 is None else [n1],
                                 None if n2 is None else [n2], albedo=(ar, ag, ab), emission=(er, eg, eb),
                                 metallic=metallic, ior=ior, rough=rough, shader=shader, alpha=alpha,
                                 uv=[(u0, v0, u1, v1, u2, v2)])
        return int(idx[0])

    def _cat(self, key: str, shape_tail=(3,), dtype=np.float64) -> np.ndarray:
        if not self._chunks:
            return np.zeros((0,) + shape_tail, dtype)
        return np.concatenate([c[key] for c in self._chunks], axis=0)

    @property
    def n_tris(self) -> int:
        return sum(len(c["p0"]) for c in self._chunks)

    def pack(self) -> PackedScene:
        n = self.n_tris
        t = np.zeros(n, _abi.TRIANGLE_DTYPE)
        for k, key in (("v0", "p0"), ("v1", "p1"), ("v2", "p2"), ("n", "n"), ("nn", "nn"), ("n0", "n0"),
                       ("n1", "n1"), ("n2", "n2")):
            t[k] = self._cat(key).astype(np.float32)
        alb = self._cat("alb")
        emi = self._cat("emi")
        t["ar"], t["ag"], t["ab"] = (alb[:, 0].astype(np.float32), alb[:, 1].astype(np.float32),
                                     alb[:, 2].astype(np.float32))
        t["er"], t["eg"], t["eb"] = (emi[:, 0].astype(np.float32), emi[:, 1].astype(np.float32),
                                     emi[:, 2].astype(np.float32))
        for key in ("ior", "rough", "metallic", "alpha"):
            t[key] = self._cat(key, ()).astype(np.float32)
        t["shader"] = self._cat("shader", (), np.int32)
        uv = self._cat("uv", (6,))
        for k, name in enumerate(("tu0", "tv0", "tu1", "tv1", "tu2", "tv2")):
            t[name] = uv[:, k].astype(np.float32)
        # textures: concatenated in order of first use (metal.mm:122-127)
        tex_ids = self._cat("texture", (), np.int32)
        t["texture_offset"] = -1
        texels = []
        offset = 0
        seen: dict[int, int] = {}
        if n and (tex_ids >= 0).any():
            first = {}
            for i in np.nonzero(tex_ids >= 0)[0]:
                first.setdefault(int(tex_ids[i]), int(i))
            for tid, _ in sorted(first.items(), key=lambda kv: kv[1]):
                seen[tid] = offset
                tex = self.textures[tid]
                texels.append(np.asarray(tex.pixels, np.float32).reshape(-1, 3))
                offset += tex.width * tex.height
            for tid, off in seen.items():
                sel = tex_ids == tid
                t["texture_offset"][sel] = off
                t["texture_width"][sel] = self.textures[tid].width
                t["texture_height"][sel] = self.textures[tid].height
        texel_arr = np.concatenate(texels).astype(np.float32) if texels else np.zeros((0, 3), np.float32)
        # emissive CDF by area x luminance (scene.cpp:73-85), accumulated in order
        light_tri = np.zeros(0, np.int32)
        cdf = np.zeros(0, np.float64)
        total = 0.0
        if n:
            s = emi[:, 0] + (emi[:, 1] + emi[:, 2])
            area2 = np.maximum(self._cat("area2", ()), 0.0)
            area = 0.5 * np.sqrt(area2)
            lit = (s > 0) & (area > 1e-12)
            light_tri = np.nonzero(lit)[0].astype(np.int32)
            lum = 0.2126 * emi[lit, 0] + 0.7152 * emi[lit, 1] + 0.0722 * emi[lit, 2]
            lum = np.maximum(lum, 1e-6)
            w = area[lit] * lum
            cdf = np.add.accumulate(w) if len(w) else w
            total = float(cdf[-1]) if len(cdf) else 0.0
        verts = np.concatenate([self._cat("p0"), self._cat("p1"), self._cat("p2")], axis=1) if n else \
            np.zeros((0, 9))
        return PackedScene(tris=t, light_tri=light_tri, light_cdf=cdf.astype(np.float32),
                           light_total=np.float32(total), texels=np.ascontiguousarray(texel_arr),
                           verts64=np.ascontiguousarray(verts))


@dataclass
class Camera:
    """raymotion::Camera (include/raymotion/pathtrace.hpp:12-52, src/engine/camera.cpp)."""
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0
    dirx: float = 0.0
    diry: float = 0.0
    dirz: float = 0.0
    fov: float = 60.0
    focal: float = 201.3839114815688
    m: tuple = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)

    @staticmethod
    def _rad(d: float) -> float:
        return d * math.pi / 180.0  # deg2rad of include/raymotion/math.hpp:17

    def update_focal(self) -> None:
        self.focal = 240.0 / math.tan(self._rad(self.fov * 0.5))

    def update_trig(self) -> None:
        r = self._rad
        cx, sx = math.cos(r(self.dirx)), math.sin(r(self.dirx))
        cy, sy = math.cos(r(self.diry)), math.sin(r(self.diry))
        cz, sz = math.cos(r(self.dirz)), math.sin(r(self.dirz))
        self.m = (cy * cz + sy * (sx * sz), -cy * sz + sy * (sx * cz), sy * cx,
                  cx * sz, cx * cz, -sx,
                  -sy * cz + cy * (sx * sz), sy * sz + cy * (sx * cz), cy * cx)

    def set(self, position=(0, 0, 0), rotation=(0, 0, 0), fov=60.0) -> "Camera":
        self.x, self.y, self.z = map(float, position)
        self.dirx, self.diry, self.dirz = map(float, rotation)
        self.fov = float(fov)
        self.update_trig()
        self.update_focal()
        return self

    def packed(self) -> _abi.RmCamera:
        c = _abi.RmCamera()
        c.x, c.y, c.z, c.focal = self.x, self.y, self.z, self.focal
        for i, v in enumerate(self.m):
            setattr(c, f"m{i}", v)
        return c


@dataclass
class RenderConfig:
    """raymotion::RenderConfig with its defaults (include/raymotion/pathtrace.hpp:54-81)."""
    width: int = 640
    height: int = 360
    spp: int = 1
    max_bounces: int = 5
    resolution: float = 1.0
    clamp: float = 16.0
    adapt_min: int = 16
    adapt_step: int = 8
    adapt_rel: float = 0.02
    adapt_abs: float = 0.002
    restir_candidates: int = 8
    restir_spatial: int = 4
    restir_radius: float = 16.0
    restir_mcap: int = 128
    flags: int = 0

    def packed(self) -> _abi.RmConfig:
        c = _abi.RmConfig()
        for f in ("width", "height", "spp", "max_bounces", "resolution", "clamp", "adapt_rel", "adapt_abs",
                  "adapt_min", "adapt_step", "restir_candidates", "restir_spatial", "restir_radius",
                  "restir_mcap", "flags"):
            setattr(c, f, getattr(self, f))
        return c
