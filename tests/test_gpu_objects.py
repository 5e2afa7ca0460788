"""Device-side scene preparation (rmcuda_model_* / rmcuda_instances_commit)
against the host path of the same step (objects.world_builder, itself pinned to
the reference's Objects::append + Scene::add_triangle in test_objects.py)."""
import numpy as np
import pytest

from raymotion_b200 import RenderError, objects
from raymotion_b200.objects import Instance
from raymotion_b200.scene import Camera, RenderConfig

from .test_objects import _instances, _model

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _check_world(backend, models, instances):
    ps = objects.world_builder(models, instances).pack()
    tris, lt, cdf, total = backend.scene_read()
    assert len(tris) == ps.n_tris
    assert tris.tobytes() == ps.tris.tobytes()
    assert np.array_equal(lt, ps.light_tri)
    assert np.array_equal(cdf, ps.light_cdf)
    assert total == ps.light_total
    return ps


def test_commit_equals_host_world_and_follows_the_refit_policy():
    """On a context of its own: the commit count that sets the rebuild
    schedule runs over the context's lifetime, as the reference's
    geometry_updates does over its Objects' (runtime.hpp:124-126)."""
    import raymotion_b200 as rb
    backend = rb.Backend(0)
    rng = np.random.default_rng(21)
    models = [_model(1, 300), _model(2, 200, emissive=True), _model(3, 150, emissive=True)]
    ids = [backend.model_create(m) for m in models]
    remap = {i: ids[i] for i in range(len(models))}
    instances = _instances(rng, len(models), 24)

    def dev(insts):
        return objects.instance_records([Instance(**{**i.__dict__, "model": remap[i.model]}) for i in insts])

    st0 = backend.stats()
    backend.instances_commit(dev(instances), rebuild_every=4)
    _check_world(backend, models, instances)
    builds, refits = 1, 0
    for step in range(1, 7):
        moved = [Instance(**{**i.__dict__, "position": tuple(np.asarray(i.position) + 0.1 * step)}) for i in instances]
        backend.instances_commit(dev(moved), rebuild_every=4)
        _check_world(backend, models, moved)
        if step % 4 == 0:
            builds += 1
        else:
            refits += 1
        st = backend.stats()
        assert (st["bvh_builds"] - st0["bvh_builds"], st["bvh_refits"] - st0["bvh_refits"]) == (builds, refits)
    # another model list: a build
    backend.instances_commit(dev(instances[:-1]), rebuild_every=4)
    _check_world(backend, models, instances[:-1])
    st = backend.stats()
    assert st["bvh_builds"] - st0["bvh_builds"] == builds + 1
    # a deforming model, same count: world re-derived
    bent = models[1].copy()
    bent["v1"] += 0.05
    backend.model_update(ids[1], bent)
    models2 = [models[0], bent, models[2]]
    backend.instances_commit(dev(instances[:-1]), rebuild_every=0)
    _check_world(backend, models2, instances[:-1])
    backend.close()


def test_rendering_a_committed_world_equals_the_uploaded_world(backend):
    torch = _torch()
    rng = np.random.default_rng(5)
    models = [_model(7, 400), _model(8, 120, emissive=True)]
    ids = [backend.model_create(m) for m in models]
    instances = _instances(rng, len(models), 16)
    for i in instances:
        i.alpha = 1.0  # opaque scene: the ReSTIR chain
    ground = objects.model_from_arrays([[-30, -3, -30], [30, -3, 30]], [[-30, -3, 30], [30, -3, -30]],
                                       [[30, -3, 30], [-30, -3, -30]], albedo=(0.5, 0.5, 0.5), rough=0.8)
    models.append(ground)
    ids.append(backend.model_create(ground))
    instances.append(Instance(model=2))
    recs = objects.instance_records(instances)
    recs["model"] = [ids[i.model] for i in instances]
    cam = Camera().set((0.0, 4.0, -22.0), (10.0, 0.0, 0.0), 60)
    cfg = RenderConfig(width=96, height=64, spp=4, max_bounces=5, restir_candidates=4, restir_spatial=2,
                       restir_radius=8.0)
    out = {}
    for how in ("host", "device"):
        backend.reset_history()
        if how == "host":
            backend.upload(objects.world_builder(models, instances).pack(), use_nodes=False)
        else:
            backend.instances_commit(recs)
        d = torch.empty(cfg.width * cfg.height * 3, dtype=torch.uint8, device="cuda")
        h = torch.empty(cfg.width * cfg.height * 3, dtype=torch.float32, device="cuda")
        backend.render_resident_async(cam, cfg, 77, d.data_ptr(), h.data_ptr())
        backend.sync()
        out[how] = (d.cpu().numpy(), h.cpu().numpy())
    assert out["host"][1].max() > 0
    assert np.array_equal(out["host"][0], out["device"][0])
    assert np.array_equal(out["host"][1].view(np.uint32), out["device"][1].view(np.uint32))


def test_invalid_instances_are_rejected(backend):
    mid = backend.model_create(_model(9, 10))
    bad = objects.instance_records([Instance(model=mid)])
    bad["model"] = 10_000
    with pytest.raises(RenderError):
        backend.instances_commit(bad)
    bad["model"] = mid
    bad["scale"] = [[1.0, 0.0, 1.0]]
    with pytest.raises(RenderError):
        backend.instances_commit(bad)
    with pytest.raises(RenderError):
        backend.model_update(mid, _model(9, 11))
