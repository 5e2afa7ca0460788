"""Instanced worlds on the host (raymotion_b200.objects) against the reference's
own Scene::add_triangle and Objects::append arithmetic (oracle/_ref, CPU)."""
import numpy as np
import pytest

from raymotion_b200 import objects
from raymotion_b200.objects import Instance


def _model(seed, n, emissive=False):
    rng = np.random.default_rng(seed)
    c = rng.normal(0, 1.0, (n, 3))
    p0 = c + rng.normal(0, 0.2, (n, 3))
    p1 = c + rng.normal(0, 0.2, (n, 3))
    p2 = c + rng.normal(0, 0.2, (n, 3))
    p2[::31] = p0[::31]  # degenerate: rejected by add_triangle
    nrm = rng.normal(0, 1, (3, n, 3))
    m = objects.model_from_arrays(p0, p1, p2, nrm[0], nrm[1], nrm[2], albedo=rng.uniform(0, 1, (n, 3)),
                                  emission=rng.uniform(0, 3, (n, 3)) * (rng.uniform(size=(n, 1)) < 0.4 if emissive else 0),
                                  metallic=rng.uniform(0, 1, n), ior=1.5, rough=rng.uniform(0, 1, n),
                                  alpha=rng.uniform(-0.2, 1.3, n), uv=rng.uniform(0, 1, (n, 6)))
    m["shader"] = rng.integers(0, 2, n)
    return m


def _instances(rng, n_models, n):
    out = []
    for _ in range(n):
        pick = rng.uniform(size=6)
        out.append(Instance(
            model=int(rng.integers(n_models)), position=tuple(rng.uniform(-10, 10, 3)),
            rotation=tuple(rng.uniform(-180, 180, 3)), scale=tuple(rng.uniform(0.3, 2.0, 3) * rng.choice([-1, 1], 3)),
            albedo=tuple(rng.uniform(0, 1, 3)) if pick[0] < 0.5 else (-1.0, -1.0, -1.0),
            emission=tuple(rng.uniform(0, 4, 3)) if pick[1] < 0.2 else (-1.0, -1.0, -1.0),
            refract=1.33 if pick[2] < 0.3 else None, rough=float(rng.uniform()) if pick[3] < 0.3 else None,
            metallic=float(rng.uniform()) if pick[4] < 0.3 else None,
            alpha=float(rng.uniform(-0.5, 1.5)) if pick[5] < 0.3 else None))
    return out


def _ref_world(ref, models, instances):
    h = ref.ref_scene_new()
    recs = objects.instance_records(instances)
    for ins, r in zip(instances, recs):
        t = models[ins.model]
        rec = np.concatenate([t["v0"], t["v1"], t["v2"],
                              np.stack([t[k] for k in ("tu0", "tv0", "tu1", "tv1", "tu2", "tv2")], axis=1),
                              t["n0"], t["n1"], t["n2"],
                              np.stack([t[k] for k in ("ar", "ag", "ab", "er", "eg", "eb", "metallic", "ior",
                                                       "rough", "alpha")], axis=1)], axis=1)
        rec = np.ascontiguousarray(rec, np.float64)
        sh = np.ascontiguousarray(t["shader"], np.int32)
        inst = np.concatenate([r["position"], np.asarray(ins.rotation, np.float64), r["scale"], r["albedo"],
                               r["emission"], [r["refract"], r["rough"], r["metallic"], r["alpha"]]])
        inst = np.ascontiguousarray(inst, np.float64)
        ref.ref_append_instance(h, rec.ctypes.data, sh.ctypes.data, len(t), inst.ctypes.data)
    return h


def test_host_world_matches_reference_objects_append(ref):
    rng = np.random.default_rng(11)
    models = [_model(1, 300), _model(2, 200, emissive=True), _model(3, 150, emissive=True)]
    instances = _instances(rng, len(models), 24)
    ps = objects.world_builder(models, instances).pack()
    h = _ref_world(ref, models, instances)
    try:
        m = ref.ref_tri_count(h)
        assert m == ps.n_tris and m > 0.9 * sum(len(models[i.model]) for i in instances)
        out = np.zeros((m, 34))
        ref.ref_tri_read(h, out.ctypes.data)
        for k, name in enumerate(("v0", "v1", "v2", "n", "nn", "n0", "n1", "n2")):
            assert np.array_equal(ps.tris[name], out[:, 3 * k:3 * k + 3].astype(np.float32)), name
        for k, name in enumerate(("ar", "ag", "ab", "er", "eg", "eb", "ior", "rough", "metallic", "alpha")):
            assert np.array_equal(ps.tris[name], out[:, 24 + k].astype(np.float32)), name
        nl = ref.ref_light_count(h)
        lt = np.zeros(nl, np.int32)
        cdf = np.zeros(nl)
        total = ref.ref_lights(h, lt.ctypes.data, cdf.ctypes.data)
        assert nl > 50
        assert np.array_equal(lt, ps.light_tri)
        assert np.array_equal(cdf.astype(np.float32), ps.light_cdf)
        assert np.float32(total) == ps.light_total
    finally:
        ref.ref_scene_free(h)


def test_instance_records_and_validation():
    recs = objects.instance_records([Instance(model=3, rotation=(90.0, 0.0, -30.0), scale=(2.0, 1.0, 1.0), rough=0.25)])
    assert recs["model"][0] == 3
    assert recs["cos_rot"][0][1] == 1.0 and recs["sin_rot"][0][1] == 0.0
    assert recs["sin_rot"][0][0] == np.sin(90.0 * np.pi / 180.0)
    assert np.isnan(recs["refract"][0]) and recs["rough"][0] == 0.25
    with pytest.raises(ValueError):
        objects.instance_records([Instance(model=0, scale=(1.0, 0.0, 1.0))])
