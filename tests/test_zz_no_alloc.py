"""rmcuda_trace_noalloc: ray queries for callers that cannot allocate device memory.

Such callers (an engine whose allocator owns the whole GPU, a fixed-budget
real-time loop, a stack that forbids runtime allocation) pass their own device
triangles, rays and output buffers; the library works in one fixed device
array.  This test calls the entry point through the C ABI twice in a row and
checks each result against rmcuda_trace on the same triangles (the resident
scene's device BVH), bit for bit as the other hit-ID tests do.  The file name
makes pytest collect it last.
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


def test_trace_noalloc_matches_trace(backend):
    import torch
    sb, cam, cfg = icosphere_field(seed=5, n_spheres=10, subdiv=3, n_emitters=64, width=96, height=54)
    scene = sb.pack()
    assert scene.n_tris <= _abi_max()
    rays = np.concatenate([camera_rays(cam, cfg, 3), random_rays(20000, [-22, -1, -22], [22, 12, 22], 9)])
    n = len(rays)
    d_rays = torch.from_numpy(rays).cuda()
    d_tris = torch.from_numpy(scene.tris.view(np.uint8)).cuda()

    def outs():
        return (torch.empty(n, dtype=torch.int32, device="cuda"), torch.empty(n, device="cuda"),
                torch.empty(n, device="cuda"), torch.empty(n, device="cuda"))

    backend.upload(scene, use_nodes=False)
    lib = _abi.load_library()
    for any_hit in (False, True):
        ref = outs()
        backend.trace(d_rays.data_ptr(), n, any_hit, *(o.data_ptr() for o in ref))
        ref = [o.cpu().numpy() for o in ref]
        for call in range(2):  # two calls in a row share the fixed array
            got = outs()
            rc, msg = _noalloc(lib, d_tris.data_ptr(), scene.n_tris, d_rays.data_ptr(), n, any_hit, got)
            assert rc == _abi.RM_OK, msg
            got = [o.cpu().numpy() for o in got]
            if any_hit:
                assert np.array_equal(got[0] >= 0, ref[0] >= 0), call
            else:
                assert np.array_equal(got[0], ref[0]), call
                hit = ref[0] >= 0
                assert hit.mean() > 0.2
                for g, r in zip(got[1:], ref[1:]):
                    assert np.array_equal(g[hit].view(np.uint32), r[hit].view(np.uint32)), call


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
