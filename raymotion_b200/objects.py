"""Instanced worlds: the reference's Objects runtime (include/raymotion/runtime.hpp:20-146).

A model is an array of object-space triangles (``_abi.MODEL_TRI_DTYPE``, the
fields of the reference's Triangle that Objects::append reads); an
``Instance`` is one Objects::push (model, position, rotation in degrees,
scale, material overrides).  ``instance_records`` turns instances into the
``rm_instance`` records of ``Backend.instances_commit``, which builds the world
on the device.  ``world_builder`` is the host path of the same step, in numpy
fp64 with the reference's operation order (Objects::append, runtime.hpp:86-113,
then Scene::add_triangle through ``SceneBuilder``): both give the same packed
triangles, light list and CDF.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from .scene import SceneBuilder


@dataclass
class Instance:
    """Objects::push arguments (runtime.hpp:76-84); negative colour components and None keep the model's."""
    model: int
    position: tuple = (0.0, 0.0, 0.0)
    rotation: tuple = (0.0, 0.0, 0.0)
    scale: tuple = (1.0, 1.0, 1.0)
    albedo: tuple = (-1.0, -1.0, -1.0)
    emission: tuple = (-1.0, -1.0, -1.0)
    refract: float | None = None
    rough: float | None = None
    metallic: float | None = None
    alpha: float | None = None


def cos_deg(d: float) -> float:
    """math.hpp:17-21: cos(d * kPi / 180) with kPi = 3.141592653589793 (= math.pi)."""
    return math.cos(d * math.pi / 180.0)


def sin_deg(d: float) -> float:
    return math.sin(d * math.pi / 180.0)


def instance_records(instances: list[Instance]) -> np.ndarray:
    """rm_instance records; the rotation's cos_deg / sin_deg are taken here, on the host."""
    out = np.zeros(len(instances), _abi.INSTANCE_DTYPE)
    for i, ins in enumerate(instances):
        if 0.0 in tuple(float(s) for s in ins.scale):
            raise ValueError("scale must be nonzero")
        r = out[i]
        r["model"] = int(ins.model)
        r["position"] = ins.position
        r["cos_rot"] = [cos_deg(float(a)) for a in ins.rotation]
        r["sin_rot"] = [sin_deg(float(a)) for a in ins.rotation]
        r["scale"] = ins.scale
        r["albedo"] = ins.albedo
        r["emission"] = ins.emission
        for k in ("refract", "rough", "metallic", "alpha"):
            v = getattr(ins, k)
            r[k] = np.nan if v is None else float(v)
    return out


def model_from_arrays(p0, p1, p2, n0=None, n1=None, n2=None, *, albedo=(1.0, 1.0, 1.0), emission=(0.0, 0.0, 0.0),
                      metallic=0.0, ior=1.0, rough=0.5, alpha=1.0, shader=0, uv=None) -> np.ndarray:
    """Object-space model triangles; per-triangle attributes broadcast.  Without
    vertex normals the face normal, normalised, is used (as for OBJ faces without vn)."""
    p0 = np.atleast_2d(np.asarray(p0, np.float64))
    p1 = np.atleast_2d(np.asarray(p1, np.float64))
    p2 = np.atleast_2d(np.asarray(p2, np.float64))
    m = len(p0)
    t = np.zeros(m, _abi.MODEL_TRI_DTYPE)
    t["v0"], t["v1"], t["v2"] = p0, p1, p2
    if n0 is None:
        e1, e2 = p1 - p0, p2 - p0
        fn = np.cross(e1, e2)
        ln = np.sqrt((fn[:, 0] * fn[:, 0] + fn[:, 1] * fn[:, 1]) + fn[:, 2] * fn[:, 2])
        fn = np.where(ln[:, None] < 1e-30, 0.0, fn / np.where(ln < 1e-30, 1.0, ln)[:, None])
        n0 = n1 = n2 = fn
    t["n0"], t["n1"], t["n2"] = n0, n1, n2
    alb = np.broadcast_to(np.asarray(albedo, np.float64), (m, 3))
    emi = np.broadcast_to(np.asarray(emission, np.float64), (m, 3))
    t["ar"], t["ag"], t["ab"] = alb[:, 0], alb[:, 1], alb[:, 2]
    t["er"], t["eg"], t["eb"] = emi[:, 0], emi[:, 1], emi[:, 2]
    t["metallic"], t["ior"], t["rough"], t["alpha"], t["shader"] = metallic, ior, rough, alpha, shader
    if uv is not None:
        uv = np.broadcast_to(np.asarray(uv, np.float64), (m, 6))
        for k, name in enumerate(("tu0", "tv0", "tu1", "tv1", "tu2", "tv2")):
            t[name] = uv[:, k]
    return t


def _rotate(c, s, v):
    """The rotate lambda of Objects::append (runtime.hpp:94-101), vectorised: x, then y, then z."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    x, y, z = x, c[0] * y - s[0] * z, s[0] * y + c[0] * z
    x, y, z = c[1] * x + s[1] * z, y, -s[1] * x + c[1] * z
    return np.stack([c[2] * x - s[2] * y, s[2] * x + c[2] * y, z], axis=1)


def _normalize(v):
    """math.hpp:58-62 (length = sqrt of dot, summed left to right)."""
    ln = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])
    small = ln < 1e-30
    return np.where(small[:, None], 0.0, v / np.where(small, 1.0, ln)[:, None])


def world_builder(models: list[np.ndarray], instances: list[Instance]) -> SceneBuilder:
    """The host path: world triangles of ``instances`` in push order, as Objects::append builds them."""
    sb = SceneBuilder()
    recs = instance_records(instances)
    for ins, r in zip(instances, recs):
        t = models[ins.model]
        if len(t) == 0:
            continue
        c, s = r["cos_rot"], r["sin_rot"]
        sc, pos = r["scale"], r["position"]

        def point(v):
            return _rotate(c, s, v * sc) + pos

        def normal(v):
            return _normalize(_rotate(c, s, v / sc))

        def pick(over, model):
            return np.where(over < 0, model, over)

        alb = np.stack([pick(r["albedo"][k], t[f]) for k, f in enumerate(("ar", "ag", "ab"))], axis=1)
        emi = np.stack([pick(r["emission"][k], t[f]) for k, f in enumerate(("er", "eg", "eb"))], axis=1)

        def opt(v, model):
            return model if np.isnan(v) else np.full(len(t), v)

        alpha = opt(r["alpha"], t["alpha"])
        alpha = np.where(np.isfinite(alpha), np.where(alpha < 0.0, 0.0, np.where(1.0 < alpha, 1.0, alpha)), 1.0)
        uv = np.stack([t[k] for k in ("tu0", "tv0", "tu1", "tv1", "tu2", "tv2")], axis=1)
        sb.add_triangles(point(t["v0"]), point(t["v1"]), point(t["v2"]), normal(t["n0"]), normal(t["n1"]),
                         normal(t["n2"]), albedo=alb, emission=emi, metallic=opt(r["metallic"], t["metallic"]),
                         ior=opt(r["refract"], t["ior"]), rough=opt(r["rough"], t["rough"]), shader=t["shader"],
                         alpha=alpha, uv=uv)
    return sb
