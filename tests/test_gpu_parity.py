"""CUDA path vs the CPU oracle on identical inputs and RNG streams (GPU)."""
import numpy as np
import pytest

from raymotion_b200 import RenderError, _abi
from raymotion_b200.scene import Camera, RenderConfig
from raymotion_b200.scenes import cornell_box, icosphere_field

from .gpu_util import camera_rays, exact_fraction, random_rays, rel_close_fraction

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _trace_gpu(backend, rays, any_hit=False):
    torch = _torch()
    r = torch.from_numpy(rays).cuda()
    n = len(rays)
    tri = torch.empty(n, dtype=torch.int32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    u = torch.empty_like(t)
    v = torch.empty_like(t)
    backend.trace(r.data_ptr(), n, any_hit, tri.data_ptr(), t.data_ptr(), u.data_ptr(), v.data_ptr())
    return tri.cpu().numpy(), t.cpu().numpy(), u.cpu().numpy(), v.cpu().numpy()


@pytest.fixture(scope="module")
def small_field(oracle):
    sb, cam, cfg = icosphere_field(seed=3, n_spheres=16, subdiv=3, n_emitters=96, width=160, height=90, spp=4,
                                   depth=6)
    sc = oracle.with_reference_bvh(sb.pack())
    return sc, cam, cfg


@pytest.mark.parametrize("use_nodes", [False, True], ids=["device_lbvh", "caller_bvh"])
def test_closest_hit_ids_bit_exact(backend, oracle, small_field, use_nodes):
    sc, cam, cfg = small_field
    backend.upload(sc, use_nodes=use_nodes)
    rays = np.concatenate([camera_rays(cam, RenderConfig(width=320, height=180), 1),
                           random_rays(40000, [-22, -1, -22], [22, 12, 22], 2)])
    g_tri, g_t, g_u, g_v = _trace_gpu(backend, rays)
    o_tri, o_t, o_u, o_v = oracle.trace(sc, rays)
    assert (o_tri >= 0).mean() > 0.2
    assert np.array_equal(g_tri, o_tri)
    hit = o_tri >= 0
    assert np.array_equal(g_t[hit].view(np.uint32), o_t[hit].view(np.uint32))
    assert np.array_equal(g_u[hit].view(np.uint32), o_u[hit].view(np.uint32))
    assert np.array_equal(g_v[hit].view(np.uint32), o_v[hit].view(np.uint32))
    g_any, _, _, _ = _trace_gpu(backend, rays, any_hit=True)
    o_any, _, _, _ = oracle.trace(sc, rays, any_hit=True)
    assert np.array_equal(g_any >= 0, o_any >= 0)


def _compare_render(backend, oracle, sc, cam, cfg, seed, use_nodes=False):
    o = oracle.Oracle()
    o_rgb, o_hdr, o_st = o.render(sc, cam, cfg, seed)
    backend.stats_reset()
    g_rgb, g_hdr = backend.render(sc, cam, cfg, seed, hdr=True, use_nodes=use_nodes)
    npix = cfg.width * cfg.height
    g_dbg = backend.debug_read(4, npix).reshape(-1, 2)
    o_dbg = o.debug_read(4, npix).reshape(-1, 2)
    st = backend.stats()
    return dict(o_rgb=o_rgb, o_hdr=o_hdr, o_st=o_st, g_rgb=g_rgb, g_hdr=g_hdr, g_dbg=g_dbg, o_dbg=o_dbg, st=st)


@pytest.mark.parametrize("spp,adapt,lanes", [(16, 16, 8), (4, 16, 1), (64, 0, 32)])
def test_cornell_plain_path_bit_exact(backend, oracle, spp, adapt, lanes):
    sb, cam, cfg = cornell_box(0)
    sc = oracle.with_reference_bvh(sb.pack())
    cfg.spp, cfg.adapt_min = spp, adapt
    r = _compare_render(backend, oracle, sc, cam, cfg, 12345)
    assert r["st"]["kernel_chain"] == lanes == r["o_st"]["chain"]
    assert np.array_equal(r["g_dbg"], r["o_dbg"]), "RNG state / sample count per pixel differ"
    assert exact_fraction(r["g_hdr"], r["o_hdr"]) == 1.0
    assert np.array_equal(r["g_rgb"], r["o_rgb"])
    assert r["st"]["path_samples"] == r["o_st"]["path_samples"]
    assert r["st"]["rays"] == r["o_st"]["rays"]


def test_field_plain_path_with_caller_bvh(backend, oracle, small_field):
    sc, cam, cfg = small_field
    cfg = RenderConfig(width=160, height=90, spp=8, max_bounces=6, adapt_min=0, restir_candidates=4,
                       restir_spatial=0)
    r = _compare_render(backend, oracle, sc, cam, cfg, 777, use_nodes=True)
    assert np.array_equal(r["g_dbg"], r["o_dbg"])
    assert exact_fraction(r["g_hdr"], r["o_hdr"]) == 1.0


def test_non_opaque_textured_nomis_norr(backend, oracle):
    from . import kat_scenes as K
    cam, cfg = K.metal_config()
    cfg.spp = 24
    cfg.flags = _abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_NOMIS | _abi.RM_FLAG_NO_RR
    sc = K.metal_scene().pack()
    sc.tris["alpha"][::3] = np.float32(0.6)
    oracle.with_reference_bvh(sc, 2)
    r = _compare_render(backend, oracle, sc, cam, cfg, 4242)
    assert np.array_equal(r["g_dbg"], r["o_dbg"])
    assert exact_fraction(r["g_hdr"], r["o_hdr"]) == 1.0


def _restir_cfg(flags=0):
    return RenderConfig(width=160, height=90, spp=4, max_bounces=6, adapt_min=0, restir_candidates=8,
                        restir_spatial=4, restir_radius=12.0, flags=flags)


@pytest.mark.parametrize("shading", ["wavefront", "wavefront-no-tail", "wavefront-all-tail", "wavefront-wide",
                                     "wavefront-split", "wavefront-one-stream", "wavefront-four-streams",
                                     "wavefront-count-wait", "megakernel"])
def test_restir_chain_matches_oracle(backend, oracle, small_field, shading, monkeypatch):
    if shading == "megakernel":
        monkeypatch.setenv("RAYMOTION_CUDA_MEGAKERNEL", "1")
    if shading == "wavefront-split":  # each traversal and shading queue in a launch of its own
        monkeypatch.setenv("RAYMOTION_CUDA_SPLIT_WAVES", "1")
    if shading == "wavefront-one-stream":  # the frame's pixels in one part, on one stream
        monkeypatch.setenv("RAYMOTION_CUDA_STREAMS", "1")
    if shading == "wavefront-four-streams":  # rows in four parts on four streams
        monkeypatch.setenv("RAYMOTION_CUDA_STREAMS", "4")
    if shading == "wavefront-count-wait":  # each batch of waves sized by a read of its own queues
        monkeypatch.setenv("RAYMOTION_CUDA_COUNT_LAG", "0")
    if shading == "wavefront-wide":
        monkeypatch.setenv("RAYMOTION_CUDA_WIDE", "1")  # every traversal on the 8-wide BVH
    # the wavefront loop hands its last paths to one tail launch; "no-tail"
    # runs waves to the end, "all-tail" hands over every path at the first read
    if shading == "wavefront-no-tail":
        monkeypatch.setenv("RAYMOTION_CUDA_TAIL", "0")
    if shading == "wavefront-all-tail":
        monkeypatch.setenv("RAYMOTION_CUDA_TAIL", "1000000000")
    sc, cam, _ = small_field
    cfg = _restir_cfg(_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_DENOISE_OFF)
    o = oracle.Oracle()
    backend.reset_history()
    npix = cfg.width * cfg.height
    for frame, seed in enumerate((11, 12)):  # the second frame reuses the first as temporal history
        o_rgb, o_hdr, o_st = o.render(sc, cam, cfg, seed)
        g_rgb, g_hdr = backend.render(sc, cam, cfg, seed, hdr=True)
        assert o_st["chain"] == 2 and backend.stats()["kernel_chain"] == 2
        og, gg = o.debug_read(0, npix), backend.debug_read(0, npix)
        assert np.array_equal(og["kind"], gg["kind"])
        live = og["kind"] != 0
        assert live.mean() > 0.3
        for f in ("pos", "normal", "albedo", "wo", "emission", "rough", "metallic", "ior"):
            assert np.array_equal(og[f][live], gg[f][live]), f
        for which in (1, 2):
            orr, grr = o.debug_read(which, npix), backend.debug_read(which, npix)
            assert np.array_equal(orr["valid"], grr["valid"])
            v = orr["valid"] != 0
            for f in ("lightPos", "lightNormal", "emission", "alpha", "p_hat", "sumWs", "sumWu", "M"):
                assert np.array_equal(orr[f][v], grr[f][v]), (which, f, frame)
        assert np.array_equal(backend.debug_read(4, npix), o.debug_read(4, npix))
        assert exact_fraction(g_hdr, o_hdr) == 1.0
        assert np.array_equal(g_rgb, o_rgb)


def test_denoiser_within_tolerance(backend, oracle, small_field):
    sc, cam, _ = small_field
    cfg = _restir_cfg(_abi.RM_FLAG_NO_ENV)
    o = oracle.Oracle()
    backend.reset_history()
    for seed in (21, 22, 23):  # frames 2 and 3 blend temporal history
        _, o_hdr, _ = o.render(sc, cam, cfg, seed)
        g_rgb, g_hdr = backend.render(sc, cam, cfg, seed, hdr=True)
        assert rel_close_fraction(g_hdr, o_hdr, 1e-4) >= 0.999


@pytest.mark.parametrize("candidates,flags", [(1, 0), (8, _abi.RM_FLAG_NOMIS), (4, _abi.RM_FLAG_NO_RR)])
def test_wavefront_shading_variants_bit_exact(backend, oracle, candidates, flags):
    """Wavefront shading vs the oracle with legacy NEE (1 candidate), MIS off and RR off."""
    sb, cam, _ = icosphere_field(seed=7, n_spheres=24, subdiv=2, n_emitters=48, width=96, height=64, spp=6, depth=7)
    sc = oracle.with_reference_bvh(sb.pack())
    cfg = RenderConfig(width=96, height=64, spp=6, max_bounces=7, adapt_min=0, restir_candidates=candidates,
                       restir_spatial=3, restir_radius=9.0, flags=_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_DENOISE_OFF | flags)
    o = oracle.Oracle()
    backend.reset_history()
    _, o_hdr, o_st = o.render(sc, cam, cfg, 99)
    _, g_hdr = backend.render(sc, cam, cfg, 99, hdr=True)
    assert o_st["chain"] == 2
    npix = cfg.width * cfg.height
    assert np.array_equal(backend.debug_read(4, npix), o.debug_read(4, npix))
    assert exact_fraction(g_hdr, o_hdr) == 1.0


def test_reupload_of_unchanged_triangles_keeps_the_bvh(backend, oracle, small_field):
    """rmcuda_render re-uploads the scene every call (metal.mm:171-186); equal
    triangles keep the device BVH (compared byte for byte on the device),
    changed ones rebuild it; the images match the oracle either way."""
    sc, cam, _ = small_field
    cfg = RenderConfig(width=64, height=40, spp=2, max_bounces=3, adapt_min=0,
                       flags=_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_RESTIR_OFF | _abi.RM_FLAG_DENOISE_OFF)
    backend.render(sc, cam, cfg, 5, use_nodes=False)
    st0 = backend.stats()
    a = backend.render(sc, cam, cfg, 5, use_nodes=False)
    st1 = backend.stats()
    assert st1["bvh_kept"] == st0["bvh_kept"] + 1 and st1["bvh_builds"] == st0["bvh_builds"]
    moved = sc.tris.copy()
    moved["v0"][::7] += np.float32(0.05)
    v64 = np.concatenate([moved["v0"], moved["v1"], moved["v2"]], axis=1).astype(np.float64)
    msc = type(sc)(tris=moved, light_tri=sc.light_tri, light_cdf=sc.light_cdf, light_total=sc.light_total,
                   texels=sc.texels, verts64=v64)
    b = backend.render(msc, cam, cfg, 5, use_nodes=False)
    st2 = backend.stats()
    assert st2["bvh_builds"] == st1["bvh_builds"] + 1 and st2["bvh_kept"] == st1["bvh_kept"]
    o_rgb, _, _ = oracle.Oracle().render(oracle.with_reference_bvh(msc), cam, cfg, 5)
    assert np.array_equal(b, o_rgb)
    assert not np.array_equal(a, b)


def test_reupload_checks_textures_against_the_new_texel_array(backend, small_field):
    """Equal triangles skip the host pass over them only when they were checked
    against the same texel count: the same textured triangles with a shorter
    texel array are still rejected, and the resident scene stays usable."""
    sc, cam, _ = small_field
    cfg = RenderConfig(width=32, height=20, spp=1, max_bounces=2, adapt_min=0,
                       flags=_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_RESTIR_OFF | _abi.RM_FLAG_DENOISE_OFF)
    tris = sc.tris.copy()
    tris["texture_offset"][0] = 0
    tris["texture_width"][0] = 2
    tris["texture_height"][0] = 2

    def scene(n_texels):
        return type(sc)(tris=tris, light_tri=sc.light_tri, light_cdf=sc.light_cdf, light_total=sc.light_total,
                        texels=np.full((n_texels, 3), 0.5, np.float32), verts64=sc.verts64)

    a = backend.render(scene(4), cam, cfg, 3, use_nodes=False)
    kept = backend.stats()["bvh_kept"]
    with pytest.raises(RenderError, match="texture outside the texel array"):
        backend.render(scene(2), cam, cfg, 3, use_nodes=False)
    b = backend.render(scene(4), cam, cfg, 3, use_nodes=False)
    assert np.array_equal(a, b)
    assert backend.stats()["bvh_kept"] >= kept + 1


def test_failed_call_drops_temporal_history(backend, small_field):
    """The reference's CacheGuard (metal.mm:105-108): a call that fails
    invalidates the temporal history, so the next ReSTIR frame renders as a
    first frame.  The failure is made on the host (a light index out of
    range), after which the scene is uploaded again unchanged."""
    sc, cam, _ = small_field
    cfg = _restir_cfg(_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_DENOISE_OFF)
    bad = type(sc)(tris=sc.tris, light_tri=np.full_like(sc.light_tri, len(sc.tris) + 5), light_cdf=sc.light_cdf,
                   light_total=sc.light_total, texels=sc.texels, verts64=sc.verts64)

    def frames(fail_between):
        backend.reset_history()
        backend.render(sc, cam, cfg, 41, use_nodes=False)
        if fail_between:
            with pytest.raises(RenderError, match="light index out of range"):
                backend.render(bad, cam, cfg, 42, use_nodes=False)
        _, hdr = backend.render(sc, cam, cfg, 43, hdr=True, use_nodes=False)
        return hdr

    with_history = frames(False)
    after_failure = frames(True)
    backend.reset_history()
    _, first = backend.render(sc, cam, cfg, 43, hdr=True, use_nodes=False)
    assert np.array_equal(after_failure.view(np.uint32), first.view(np.uint32))
    assert not np.array_equal(with_history.view(np.uint32), first.view(np.uint32))


@pytest.mark.parametrize("shading", ["wavefront", "megakernel"])
def test_restir_chain_on_a_textured_scene_matches_oracle(backend, oracle, shading, monkeypatch):
    """The ReSTIR chain (generate, temporal + spatial reuse, shade, denoiser
    off) on the known-answer scene with its 2x2 texture on walls, metal and
    both dielectrics (nearest sampling with wrap, pathtrace.metal:178-185):
    bit-exact radiance over two frames, the second with temporal history."""
    from . import kat_scenes as K
    if shading == "megakernel":
        monkeypatch.setenv("RAYMOTION_CUDA_MEGAKERNEL", "1")
    cam, _ = K.metal_config()
    cfg = RenderConfig(width=96, height=64, spp=8, max_bounces=6, adapt_min=0, restir_candidates=8,
                       restir_spatial=3, restir_radius=8.0, flags=_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_DENOISE_OFF)
    sc = K.metal_scene().pack()
    assert (sc.tris["texture_offset"] >= 0).any()
    oracle.with_reference_bvh(sc, 2)
    o = oracle.Oracle()
    backend.reset_history()
    for seed in (5, 6):
        _, o_hdr, o_st = o.render(sc, cam, cfg, seed)
        _, g_hdr = backend.render(sc, cam, cfg, seed, hdr=True)
        assert o_st["chain"] == 2 and backend.stats()["kernel_chain"] == 2
        assert o_hdr.max() > 0
        assert exact_fraction(g_hdr, o_hdr) == 1.0


def test_speculative_reupload_frames_equal_plain_frames(backend, small_field, monkeypatch):
    """rmcuda_render renders an unchanged re-upload while the triangles are
    sent and compared on a second stream; when they differ, the speculative
    frame is undone (temporal history, counters) and the upload rendered the
    ordinary way.  A ReSTIR sequence over static, then moved, then static
    triangles gives the same radiance, sample counts and BVH builds with
    speculation on and off."""
    sc, cam, _ = small_field
    cfg = _restir_cfg(_abi.RM_FLAG_NO_ENV)
    moved = sc.tris.copy()
    moved["v0"][::5] += np.float32(0.03)
    v64 = np.concatenate([moved["v0"], moved["v1"], moved["v2"]], axis=1).astype(np.float64)
    msc = type(sc)(tris=moved, light_tri=sc.light_tri, light_cdf=sc.light_cdf, light_total=sc.light_total,
                   texels=sc.texels, verts64=v64)
    tiny = type(sc)(tris=sc.tris[:3], light_tri=sc.light_tri[:0], light_cdf=sc.light_cdf[:0], light_total=0.0,
                    texels=sc.texels, verts64=sc.verts64[:3])
    frames = [sc, sc, sc, msc, msc, msc, sc, sc]

    def run(speculate):
        monkeypatch.setenv("RAYMOTION_CUDA_SPECULATE", "1" if speculate else "0")
        backend.upload(tiny, use_nodes=False)  # another resident scene first
        backend.reset_history()
        backend.stats_reset()
        st0 = backend.stats()
        out = []
        for k, s in enumerate(frames):
            _, hdr = backend.render(s, cam, cfg, 70 + k, hdr=True, use_nodes=False)
            st = backend.stats()
            out.append((hdr.copy(), st["path_samples"], st["bvh_builds"] - st0["bvh_builds"]))
        return out

    on, off = run(True), run(False)
    for k, ((h1, s1, b1), (h0, s0, b0)) in enumerate(zip(on, off)):
        assert np.array_equal(h1.view(np.uint32), h0.view(np.uint32)), k
        assert s1 == s0 and b1 == b0, (k, s1, s0, b1, b0)
    assert on[-1][2] == 3  # built for the first frame, the moved triangles and their return


@pytest.mark.parametrize("parts,height", [(4, 3), (3, 7), (2, 1)])
def test_wavefront_parts_with_few_rows(backend, oracle, small_field, parts, height, monkeypatch):
    """Frames whose height is below or not a multiple of the number of row
    parts (fewer rows than parts run as one part): bit-exact radiance, RNG
    state and sample counts."""
    monkeypatch.setenv("RAYMOTION_CUDA_STREAMS", str(parts))
    sc, cam, _ = small_field
    cfg = RenderConfig(width=96, height=height, spp=4, max_bounces=6, adapt_min=0, restir_candidates=8,
                       restir_spatial=4, restir_radius=12.0, flags=_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_DENOISE_OFF)
    o = oracle.Oracle()
    backend.reset_history()
    _, o_hdr, o_st = o.render(sc, cam, cfg, 31)
    _, g_hdr = backend.render(sc, cam, cfg, 31, hdr=True)
    assert o_st["chain"] == 2 and backend.stats()["kernel_chain"] == 2
    npix = cfg.width * cfg.height
    assert np.array_equal(backend.debug_read(4, npix), o.debug_read(4, npix))
    assert exact_fraction(g_hdr, o_hdr) == 1.0
