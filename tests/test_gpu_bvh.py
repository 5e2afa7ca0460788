"""Device BVH builds (PLOC clustering, LBVH), caller-BVH conversion and device
refit / rebuild: closest hits stay bit-identical to the oracle's (GPU)."""
import numpy as np
import pytest

from raymotion_b200.scene import SceneBuilder
from raymotion_b200.scenes import icosphere_field

from .gpu_util import random_rays
from .test_gpu_parity import _trace_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def field(oracle):
    sb, cam, cfg = icosphere_field(seed=11, n_spheres=20, subdiv=3, n_emitters=32, width=64, height=36)
    return sb.pack()


def _check_hits(backend, oracle, scene, rays):
    g_tri, g_t, _, _ = _trace_gpu(backend, rays)
    o_tri, o_t, _, _ = oracle.trace(scene, rays)
    assert np.array_equal(g_tri, o_tri)
    hit = o_tri >= 0
    assert np.array_equal(g_t[hit].view(np.uint32), o_t[hit].view(np.uint32))
    return hit.mean()


@pytest.mark.parametrize("builder,leaf", [("ploc", "4"), ("ploc", "1"), ("ploc", "8"), ("lbvh", "4")])
def test_device_builders_give_identical_hits(backend, oracle, field, builder, leaf, monkeypatch):
    monkeypatch.setenv("RAYMOTION_CUDA_BVH", builder)
    monkeypatch.setenv("RAYMOTION_CUDA_BVH_LEAF", leaf)
    sc = oracle.with_reference_bvh(field)
    backend.upload(sc, use_nodes=False)
    rays = random_rays(30000, [-22, -1, -22], [22, 12, 22], 5)
    assert _check_hits(backend, oracle, sc, rays) > 0.2


def test_device_bvh_quality_near_the_reference_sah_bvh(backend, oracle, field, monkeypatch):
    """Hits do not depend on the BVH, so a correct tree over a badly ordered
    build (a broken Morton sort, say) would pass every hit test; its node
    visits per ray would not.  The device builds stay near the reference's SAH
    BVH (converted) on the same frame."""
    from raymotion_b200 import _abi
    _, cam, cfg = icosphere_field(seed=11, n_spheres=20, subdiv=3, n_emitters=32, width=64, height=36)
    cfg.flags = _abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_DENOISE_OFF
    sc = oracle.with_reference_bvh(field)
    per_ray = {}
    for name, use_nodes, builder in (("sah", True, "ploc"), ("ploc", False, "ploc"), ("lbvh", False, "lbvh")):
        monkeypatch.setenv("RAYMOTION_CUDA_BVH", builder)
        backend.stats_reset()
        backend.render(sc, cam, cfg, 7, use_nodes=use_nodes)
        st = backend.stats()
        assert st["rays"] > 10000
        per_ray[name] = st["nodes_visited"] / st["rays"]
    assert per_ray["ploc"] < 2.0 * per_ray["sah"], per_ray
    assert per_ray["lbvh"] < 3.0 * per_ray["sah"], per_ray


def test_degenerate_clusters(backend, oracle):
    """300 copies of one triangle: no mutual nearest neighbours by area ties; the
    build must still terminate, and ties resolve to the smallest index."""
    sb = SceneBuilder()
    p = np.array([[0.0, 0.0, 3.0]] * 300)
    sb.add_triangles(p + [-1, -1, 0], p + [1, -1, 0], p + [0, 1, 0])
    sc = oracle.with_reference_bvh(sb.pack())
    backend.upload(sc, use_nodes=False)
    rays = random_rays(2000, [-0.5, -0.5, -1], [0.5, 0.5, 0], 2)
    rays[:, 3:6] = [0, 0, 1]
    g_tri, _, _, _ = _trace_gpu(backend, rays)
    o_tri, _, _, _ = oracle.trace(sc, rays)
    assert np.array_equal(g_tri, o_tri)
    assert (o_tri[o_tri >= 0] == 0).all()


def _moved(scene, shift):
    moved = scene.tris.copy()
    for f in ("v0", "v1", "v2"):
        moved[f][: len(moved) // 2] += np.float32(shift)
    return moved


@pytest.mark.parametrize("use_nodes", [False, True], ids=["device_bvh", "caller_bvh"])
def test_refit_and_rebuild_track_moved_geometry(backend, oracle, field, use_nodes):
    sc = oracle.with_reference_bvh(field)
    backend.upload(sc, use_nodes=use_nodes)
    rays = random_rays(30000, [-22, -1, -22], [22, 12, 22], 8)
    for step, (shift, rebuild_every) in enumerate([((0.7, 0.3, -0.4), 0), ((-1.1, 0.2, 0.9), 0), ((0.2, 2.0, 0.1), 1)]):
        moved = _moved(sc, shift)
        backend.update(moved, rebuild_every=rebuild_every)
        ms = oracle.with_reference_bvh(type(sc)(tris=moved, light_tri=sc.light_tri, light_cdf=sc.light_cdf,
                                                light_total=sc.light_total, texels=sc.texels,
                                                verts64=np.concatenate([moved["v0"], moved["v1"], moved["v2"]],
                                                                       axis=1).astype(np.float64)))
        assert _check_hits(backend, oracle, ms, rays) > 0.2, step


@pytest.mark.parametrize("builder", ["ploc", "lbvh"])
def test_wide_bvh_hits_equal_binary_and_oracle(backend, oracle, field, builder, monkeypatch):
    """The 8-wide compressed BVH (collapsed from the device build) answers
    closest-hit and any-hit queries exactly as the binary BVH and the oracle,
    also after a refit, whose records it is collapsed again from."""
    monkeypatch.setenv("RAYMOTION_CUDA_BVH", builder)
    sc = oracle.with_reference_bvh(field)
    rays = np.concatenate([random_rays(30000, [-22, -1, -22], [22, 12, 22], 7),
                           random_rays(5000, [-22, -1, -22], [22, 12, 22], 8, tmax=3.0)])
    out = {}
    for wide in ("1", "0"):
        monkeypatch.setenv("RAYMOTION_CUDA_WIDE", wide)
        backend.upload(sc, use_nodes=False)
        backend.render(sc, *_tiny_view(), use_nodes=False)  # stats come from the resident scene
        assert backend.stats()["bvh_node_bytes"] == (80 if wide == "1" else 64)
        out[wide] = (_trace_gpu(backend, rays), _trace_gpu(backend, rays, any_hit=True))
    (w_tri, w_t, w_u, w_v), (w_any, _, _, _) = out["1"]
    (b_tri, b_t, b_u, b_v), (b_any, _, _, _) = out["0"]
    hit = b_tri >= 0
    assert hit.mean() > 0.2
    assert np.array_equal(w_tri, b_tri)
    for a, b in ((w_t, b_t), (w_u, b_u), (w_v, b_v)):
        assert np.array_equal(a[hit].view(np.uint32), b[hit].view(np.uint32))
    assert np.array_equal(w_any >= 0, b_any >= 0)
    assert _check_hits(backend, oracle, sc, rays) > 0.2
    # moved geometry: refit, then the wide nodes are collapsed again
    monkeypatch.setenv("RAYMOTION_CUDA_WIDE", "1")
    backend.upload(sc, use_nodes=False)
    moved = _moved(sc, 0.37)
    backend.update(moved, rebuild_every=0)
    msc = oracle.with_reference_bvh(type(sc)(tris=moved, light_tri=sc.light_tri, light_cdf=sc.light_cdf,
                                              light_total=sc.light_total, texels=sc.texels,
                                              verts64=_verts64(moved)))
    assert _check_hits(backend, oracle, msc, rays) > 0.2


def _tiny_view():
    from raymotion_b200.scene import Camera, RenderConfig
    cam = Camera().set((0.0, 9.0, -34.0), (14.0, 0.0, 0.0), 60)
    return cam, RenderConfig(width=8, height=8, spp=1, max_bounces=1)


def _verts64(tris):
    return np.concatenate([tris["v0"], tris["v1"], tris["v2"]], axis=1).astype(np.float64)
