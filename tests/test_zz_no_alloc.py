"""rmcuda_trace_noalloc: ray queries for callers that cannot allocate device memory.

Such callers (an engine whose allocator owns the whole GPU, a fixed-budget
real-time loop, a stack that forbids runtime allocation) pass their own device
triangles, rays and output buffers; the library works in one fixed device
array.  These tests call the entry point through the C ABI, two calls in a row
where the array is shared, and check each result against rmcuda_trace on the
same triangles (the resident scene's device BVH) and against the CPU oracle,
bit for bit as the other hit-ID tests do: a mid-size scene, an empty scene
right after a full one (the array keeps the last call's contents), scenes of
one to four triangles (a single leaf) and a scene at the size limit.  The file
name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from raymotion_b200 import _abi
from raymotion_b200.scenes import icosphere_field

from .gpu_util import camera_rays, random_rays

pytestmark = pytest.mark.gpu


def _noalloc(lib, d_tris, n_tris, d_rays, n_rays, any_hit, outs):
    err = C.create_string_buffer(512)
    tri, t, u, v = outs
    rc = lib.rmcuda_trace_noalloc(d_tris, n_tris, d_rays, n_rays, int(any_hit), tri.data_ptr(), t.data_ptr(),
                                  u.data_ptr(), v.data_ptr(), None, err, 512)
    return rc, err.value.decode()


def _outs(n):
    import torch
    return (torch.empty(n, dtype=torch.int32, device="cuda"), torch.empty(n, device="cuda"),
            torch.empty(n, device="cuda"), torch.empty(n, device="cuda"))


def _run(lib, scene, d_rays, n, any_hit):
    import torch
    d_tris = torch.from_numpy(scene.tris.view(np.uint8).copy()).cuda() if scene.n_tris else None
    got = _outs(n)
    rc, msg = _noalloc(lib, d_tris.data_ptr() if d_tris is not None else None, scene.n_tris, d_rays.data_ptr(), n,
                       any_hit, got)
    assert rc == _abi.RM_OK, msg
    return [o.cpu().numpy() for o in got]


def _same_hits(got, ref, any_hit, what):
    if any_hit:
        assert np.array_equal(got[0] >= 0, ref[0] >= 0), what
        return
    assert np.array_equal(got[0], ref[0]), what
    hit = ref[0] >= 0
    for g, r in zip(got[1:], ref[1:]):
        assert np.array_equal(g[hit].view(np.uint32), r[hit].view(np.uint32)), what


def _field_rays(cam, cfg, n_random, seed):
    return np.concatenate([camera_rays(cam, cfg, seed), random_rays(n_random, [-22, -1, -22], [22, 12, 22], seed)])


def test_trace_noalloc_matches_trace(backend):
    import torch
    sb, cam, cfg = icosphere_field(seed=5, n_spheres=10, subdiv=3, n_emitters=64, width=96, height=54)
    scene = sb.pack()
    assert scene.n_tris <= _abi_max()
    rays = _field_rays(cam, cfg, 20000, 9)
    n = len(rays)
    d_rays = torch.from_numpy(rays).cuda()
    backend.upload(scene, use_nodes=False)
    lib = _abi.load_library()
    for any_hit in (False, True):
        ref = _outs(n)
        backend.trace(d_rays.data_ptr(), n, any_hit, *(o.data_ptr() for o in ref))
        ref = [o.cpu().numpy() for o in ref]
        assert (ref[0] >= 0).mean() > 0.2
        for call in range(2):  # two calls in a row share the fixed array
            _same_hits(_run(lib, scene, d_rays, n, any_hit), ref, any_hit, call)


def test_trace_noalloc_matches_oracle_and_an_empty_scene_after_a_full_one(backend, oracle):
    """Hit IDs, t, u and v equal the oracle's traversal of the reference's own
    BVH; a zero-triangle call right after it reports every ray a miss and no
    error, whatever the previous call left in the shared array."""
    import torch
    sb, cam, cfg = icosphere_field(seed=6, n_spheres=8, subdiv=3, n_emitters=40, width=80, height=45)
    scene = oracle.with_reference_bvh(sb.pack())
    rays = _field_rays(cam, cfg, 8000, 4)
    n = len(rays)
    d_rays = torch.from_numpy(rays).cuda()
    lib = _abi.load_library()
    o_tri, o_t, o_u, o_v = oracle.trace(scene, rays)
    assert (o_tri >= 0).mean() > 0.2
    got = _run(lib, scene, d_rays, n, False)
    _same_hits(got, [o_tri, o_t, o_u, o_v], False, "oracle")
    empty = type(scene)(tris=scene.tris[:0], light_tri=scene.light_tri[:0], light_cdf=scene.light_cdf[:0],
                        light_total=0.0, texels=scene.texels, verts64=scene.verts64[:0])
    for any_hit in (False, True):
        tri = _run(lib, empty, d_rays, n, any_hit)[0]
        assert (tri == -1).all(), any_hit


@pytest.mark.parametrize("n_tris", [1, 2, 3, 4])
def test_trace_noalloc_single_leaf_scenes(backend, oracle, n_tris):
    """Up to four triangles form one leaf (no sort, no tree): equal to the oracle."""
    import torch
    sb, cam, cfg = icosphere_field(seed=8, n_spheres=2, subdiv=0, n_emitters=8, width=64, height=36)
    full = sb.pack()
    pick = np.random.default_rng(n_tris).choice(full.n_tris, n_tris, replace=False)
    tris = full.tris[pick]
    v64 = full.verts64[pick]
    scene = type(full)(tris=tris, light_tri=np.zeros(0, np.int32), light_cdf=np.zeros(0, np.float32),
                       light_total=0.0, texels=full.texels, verts64=v64)
    oracle.with_reference_bvh(scene)
    # rays aimed at the chosen triangles' centroids from random origins, plus random rays
    rng = np.random.default_rng(100 + n_tris)
    cen = v64.reshape(-1, 3, 3).mean(axis=1)
    o = rng.uniform([-22, -1, -22], [22, 12, 22], (3000, 3))
    d = cen[rng.integers(0, n_tris, 3000)] - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    aimed = np.zeros((3000, 7), np.float32)
    aimed[:, :3], aimed[:, 3:6], aimed[:, 6] = o, d, 1e30
    rays = np.concatenate([aimed, random_rays(2000, [-22, -1, -22], [22, 12, 22], n_tris)])
    d_rays = torch.from_numpy(rays).cuda()
    lib = _abi.load_library()
    ref = list(oracle.trace(scene, rays))
    assert (ref[0] >= 0).mean() > 0.3
    for any_hit in (False, True):
        if any_hit:
            ref = list(oracle.trace(scene, rays, any_hit=True))
        for call in range(2):
            _same_hits(_run(lib, scene, d_rays, len(rays), any_hit), ref, any_hit, (any_hit, call))


def test_trace_noalloc_at_the_size_limit(backend):
    """A scene of exactly RMCUDA_NOALLOC_MAX_TRIS triangles fits the fixed
    array and answers like rmcuda_trace (one more is rejected, below)."""
    import torch
    limit = _abi_max()
    per_sphere = 1280  # subdivision 3
    n_spheres = (limit - 2 - 64) // per_sphere
    n_emitters = limit - 2 - n_spheres * per_sphere
    sb, cam, cfg = icosphere_field(seed=9, n_spheres=n_spheres, subdiv=3, n_emitters=n_emitters, width=96,
                                   height=54)
    scene = sb.pack()
    assert scene.n_tris == limit, scene.n_tris
    rays = _field_rays(cam, cfg, 20000, 11)
    n = len(rays)
    d_rays = torch.from_numpy(rays).cuda()
    backend.upload(scene, use_nodes=False)
    lib = _abi.load_library()
    ref = _outs(n)
    backend.trace(d_rays.data_ptr(), n, False, *(o.data_ptr() for o in ref))
    ref = [o.cpu().numpy() for o in ref]
    for call in range(2):
        _same_hits(_run(lib, scene, d_rays, n, False), ref, False, call)


def test_trace_noalloc_rejects_oversized_scenes():
    lib = _abi.load_library()
    err = C.create_string_buffer(512)
    rc = lib.rmcuda_trace_noalloc(C.c_void_p(16), _abi_max() + 1, C.c_void_p(16), 1, 0, C.c_void_p(16), None, None,
                                  None, None, err, 512)
    assert rc == _abi.RM_ERR_INVALID
    assert b"exceed the maximum" in err.value


def _abi_max():
    import re
    from pathlib import Path
    text = (Path(__file__).resolve().parents[1] / "include" / "rmcuda.h").read_text()
    return int(re.search(r"#define RMCUDA_NOALLOC_MAX_TRIS (\d+)", text).group(1))
