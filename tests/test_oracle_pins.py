"""Pin the oracle and the caller-side scene model against the reference's own
CPU code (oracle/_ref/libref.so = src/engine/{scene,bvh,camera}.cpp)."""
import numpy as np
import pytest

from raymotion_b200.scene import Camera, SceneBuilder
from raymotion_b200.scenes import cornell_box


def _random_soup(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform([-20, 0, -20], [20, 10, 20], (n, 3))
    p0 = c + rng.normal(0, 0.3, (n, 3))
    p1 = c + rng.normal(0, 0.3, (n, 3))
    p2 = c + rng.normal(0, 0.3, (n, 3))
    return p0, p1, p2


def _ref_scene(ref, sb_calls):
    import ctypes as C
    h = ref.ref_scene_new()
    for rec, shader in sb_calls:
        r = np.ascontiguousarray(rec, np.float64)
        ref.ref_add_triangle(h, r.ctypes.data, shader)
    return h


def _records(p0, p1, p2, emis, alpha):
    recs = []
    for i in range(len(p0)):
        n = np.cross(p1[i] - p0[i], p2[i] - p0[i])
        rec = np.concatenate([p0[i], p1[i], p2[i], np.zeros(6), n, n, n, [0.5, 0.6, 0.7], emis[i],
                              [0.25, 1.5, 0.4, alpha[i]]])
        recs.append((rec, 0))
    return recs


def test_scene_builder_matches_reference_add_triangle(ref):
    n = 600
    p0, p1, p2 = _random_soup(n, 3)
    p2[::97] = p0[::97]  # degenerate triangles are rejected
    rng = np.random.default_rng(4)
    emis = np.where(rng.uniform(size=(n, 1)) < 0.3, rng.uniform(0, 5, (n, 3)), 0.0)
    alpha = rng.uniform(-0.5, 1.5, n)
    sb = SceneBuilder()
    for i in range(n):
        nrm = np.cross(p1[i] - p0[i], p2[i] - p0[i])
        sb.add_triangles([p0[i]], [p1[i]], [p2[i]], [nrm], [nrm], [nrm], albedo=(0.5, 0.6, 0.7), emission=emis[i],
                         metallic=0.25, ior=1.5, rough=0.4, alpha=alpha[i])
    ps = sb.pack()
    h = _ref_scene(ref, _records(p0, p1, p2, emis, alpha))
    try:
        m = ref.ref_tri_count(h)
        assert m == ps.n_tris
        out = np.zeros((m, 34))
        ref.ref_tri_read(h, out.ctypes.data)
        # fp32 packing of the reference triangle equals our packing, field for field
        for k, name in enumerate(("v0", "v1", "v2", "n", "nn", "n0", "n1", "n2")):
            assert np.array_equal(ps.tris[name], out[:, 3 * k:3 * k + 3].astype(np.float32)), name
        assert np.array_equal(ps.tris["alpha"], out[:, 33].astype(np.float32))
        nl = ref.ref_light_count(h)
        lt = np.zeros(nl, np.int32)
        cdf = np.zeros(nl)
        total = ref.ref_lights(h, lt.ctypes.data, cdf.ctypes.data)
        assert np.array_equal(lt, ps.light_tri)
        assert np.array_equal(cdf.astype(np.float32), ps.light_cdf)
        assert np.float32(total) == ps.light_total
    finally:
        ref.ref_scene_free(h)


@pytest.mark.parametrize("n,leaf,seed", [(36, 8, 0), (40, 2, 1), (3000, 8, 2), (2500, 4, 5)])
def test_oracle_bvh_equals_reference_bvh(ref, oracle, n, leaf, seed):
    if n == 36:
        sb, _, _ = cornell_box(0)
        ps = sb.pack()
        verts = ps.verts64
    else:
        p0, p1, p2 = _random_soup(n, seed)
        verts = np.concatenate([p0, p1, p2], axis=1)
    recs = []
    for v in verts:
        nrm = np.cross(v[3:6] - v[0:3], v[6:9] - v[0:3])
        recs.append((np.concatenate([v, np.zeros(6), nrm, nrm, nrm, [1, 1, 1, 0, 0, 0, 0, 1, .5, 1]]), 0))
    h = _ref_scene(ref, recs)
    try:
        assert ref.ref_tri_count(h) == len(verts)
        m = ref.ref_build_bvh(h, leaf)
        rb = np.zeros((m, 6))
        rl = np.zeros((m, 4), np.int32)
        ro = np.zeros(len(verts), np.int32)
        ref.ref_nodes(h, rb.ctypes.data, rl.ctypes.data, ro.ctypes.data)
        ob, ol, oo = oracle.build_bvh(verts, leaf)
        assert np.array_equal(rb, ob)
        assert np.array_equal(rl, ol)
        assert np.array_equal(ro, oo)
        # refit after moving every vertex: reverse-order refit agrees too
        moved = verts + np.array([0.3, -0.2, 0.1] * 3)
        ref.ref_move_vertices(h, np.ascontiguousarray(moved).ctypes.data)
        ref.ref_refit_bvh(h)
        ref.ref_nodes(h, rb.ctypes.data, rl.ctypes.data, ro.ctypes.data)
        assert np.array_equal(rb, oracle.refit_bvh(moved, ob, ol, oo))
    finally:
        ref.ref_scene_free(h)


def test_refit_known_answers(oracle):
    """reference tests/test_bvh.cpp:13-24 restated on the oracle BVH."""
    def fill(z, n):
        x = np.arange(n) * 3.0
        return np.stack([x - 1, -np.ones(n), np.full(n, z), x + 1, -np.ones(n), np.full(n, z), x, np.ones(n),
                         np.full(n, z)], axis=1)
    b, l, o = oracle.build_bvh(fill(3, 40), 2)
    moved = fill(7, 40)
    r = oracle.refit_bvh(moved, b, l, o)
    assert r[0, 2] == 7 and r[0, 5] == 7
    rb, _, _ = oracle.build_bvh(moved, 2)
    assert r[0, 0] == rb[0, 0] and r[0, 3] == rb[0, 3]
    b1, l1, o1 = oracle.build_bvh(fill(9, 1), 2)
    assert b1[0, 2] == 9 and len(o1) == 1
    b0, _, _ = oracle.build_bvh(np.zeros((0, 9)), 2)
    assert len(b0) == 0


@pytest.mark.parametrize("pos,rot,fov", [((0, 0, 0), (0, 0, 0), 60), ((1, 2, -3), (14, -33, 7), 52),
                                         ((0, 9, -34), (14, 0, 0), 106)])
def test_camera_matches_reference(ref, pos, rot, fov):
    out = np.zeros(10)
    ref.ref_camera(*pos, *rot, fov, out.ctypes.data)
    cam = Camera().set(pos, rot, fov)
    assert cam.focal == out[0]
    assert np.array_equal(np.asarray(cam.m), out[1:])
