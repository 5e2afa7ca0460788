"""Parity on the configurations the benchmark runs (GPU).

* The headline frame exactly as benchmarked: the 1,028,098-triangle icosphere
  field at 1280x720, 64 spp (32 lanes), depth 12, ReSTIR DI with 32 RIS
  candidates, 5 spatial neighbours in a 30 px square, temporal reuse, the
  denoiser on and the device PLOC BVH.  The GPU renders two whole frames
  through rmcuda_render; the oracle renders bands of rows of the same two
  frames (its generate pass pads each band by the spatial radius, and the
  first frame's band is wider than the second's, so every temporal lookup of
  the second band reads history the oracle computed).  On each band: G-buffer,
  initial and merged reservoirs, per-pixel RNG state and sample count, and the
  shaded radiance are bit-exact; the denoised radiance is within 1e-4
  relative on >= 99.9 % of the band's interior pixels (the a-trous filter is
  the one stage compiled with fused multiply-adds).  One band sits mid-frame,
  one at the bottom edge (the ground; the top rows are sky), where the 30 px
  neighbour square leaves the frame.
* Config 0 as stated: the Cornell box at 320x180, 16 spp, depth 8, NEE + MIS,
  Russian roulette off (RM_FLAG_NO_RR), bit-exact over the whole frame.
* Temporal reuse on animated geometry (RM_FLAG_ANIMATED_HISTORY, the
  animated sequence's mode): moving instances, a deforming cloth and an
  orbiting camera, the world committed on the device and refitted; three
  frames against the oracle rendering the host-built world of each frame.
"""
import numpy as np
import pytest

from raymotion_b200 import _abi, objects
from raymotion_b200.scenes import AnimatedSequence, cornell_box, icosphere_field

from .gpu_util import exact_fraction, rel_close_fraction

pytestmark = pytest.mark.gpu

GB_FIELDS = ("pos", "normal", "albedo", "wo", "emission", "rough", "metallic", "ior")
RES_FIELDS = ("lightPos", "lightNormal", "emission", "alpha", "p_hat", "sumWs", "sumWu", "M")
SEEDS = (12345, 12346)
# frame 1 band = frame 2 band widened by this many rows on each side: temporal
# reprojection of a static camera moves at most a pixel, the denoiser reaches
# +-7 rows (3x3 clamp, a-trous strides 1 and 2)
HIST_MARGIN = 16
DENOISE_REACH = 8


def _frame_buffers(src, npix):
    return dict(g=src.debug_read(0, npix), r_init=src.debug_read(1, npix), r_merged=src.debug_read(2, npix),
                hdr_shaded=src.debug_read(3, npix), dbg=src.debug_read(4, npix))


def _compare_band(gpu, orc, W, r0, r1, what):
    sl = slice(r0 * W, r1 * W)
    og, gg = orc["g"][sl], gpu["g"][sl]
    assert np.array_equal(og["kind"], gg["kind"]), what
    live = og["kind"] != 0
    assert live.mean() > 0.3, what
    for f in GB_FIELDS:
        assert np.array_equal(og[f][live], gg[f][live]), (what, f)
    for key in ("r_init", "r_merged"):
        orr, grr = orc[key][sl], gpu[key][sl]
        assert np.array_equal(orr["valid"], grr["valid"]), (what, key)
        v = orr["valid"] != 0
        assert v.mean() > 0.2, (what, key)
        for f in RES_FIELDS:
            assert np.array_equal(orr[f][v], grr[f][v]), (what, key, f)
    assert np.array_equal(orc["dbg"][2 * r0 * W:2 * r1 * W], gpu["dbg"][2 * r0 * W:2 * r1 * W]), (what, "rng/samples")
    oh, gh = orc["hdr_shaded"][3 * r0 * W:3 * r1 * W], gpu["hdr_shaded"][3 * r0 * W:3 * r1 * W]
    assert oh.max() > 0, what
    assert exact_fraction(gh, oh) == 1.0, (what, "shaded radiance")


@pytest.fixture(scope="module")
def headline(backend, oracle):
    """The benchmarked frame and the GPU's two frames of it (whole frames)."""
    sb, cam, cfg = icosphere_field(seed=1)
    assert (cfg.width, cfg.height, cfg.spp, cfg.max_bounces) == (1280, 720, 64, 12)
    assert (cfg.restir_candidates, cfg.restir_spatial, cfg.restir_radius) == (32, 5, 30.0)
    cfg.flags = _abi.RM_FLAG_NO_ENV  # ReSTIR, temporal reuse and the denoiser on, as benchmarked
    scene = sb.pack()
    assert scene.n_tris == 1_028_098
    npix = cfg.width * cfg.height
    backend.reset_history()
    frames = []
    for seed in SEEDS:
        rgb, hdr = backend.render(scene, cam, cfg, seed, hdr=True, use_nodes=False)  # device PLOC BVH
        st = backend.stats()
        assert st["kernel_chain"] == 2
        frames.append(dict(_frame_buffers(backend, npix), hdr_final=hdr, rgb=rgb))
    oracle.with_reference_bvh(scene)
    return scene, cam, cfg, frames


@pytest.mark.parametrize("band", [(352, 376), (696, 720)], ids=["mid_frame", "bottom_edge"])
def test_headline_frame_matches_oracle_on_a_band(oracle, headline, band):
    scene, cam, cfg, gpu = headline
    W, H = cfg.width, cfg.height
    npix = W * H
    r0, r1 = band
    o = oracle.Oracle()
    bands = [(max(0, r0 - HIST_MARGIN), min(H, r1 + HIST_MARGIN)), (r0, r1)]
    for k, (seed, (b0, b1)) in enumerate(zip(SEEDS, bands)):
        _, o_hdr, o_st = o.render(scene, cam, cfg, seed, rows=(b0, b1))
        assert o_st["chain"] == 2
        orc = _frame_buffers(o, npix)
        _compare_band(gpu[k], orc, W, b0, b1, f"frame {k + 1} rows {b0}..{b1 - 1}")
        # the denoised output, away from the band's cut edges
        d0 = b0 if b0 == 0 else b0 + DENOISE_REACH
        d1 = b1 if b1 == H else b1 - DENOISE_REACH
        oh, gh = o_hdr[3 * d0 * W:3 * d1 * W], gpu[k]["hdr_final"][3 * d0 * W:3 * d1 * W]
        assert oh.max() > 0
        assert rel_close_fraction(gh, oh, 1e-4) >= 0.999, (k, d0, d1)


@pytest.mark.parametrize("rr", [False, True], ids=["rr_off_config0", "rr_on"])
def test_config0_cornell_box_as_stated(backend, oracle, rr):
    """Config 0: 36 triangles, 320x180, 16 spp (8 lanes of 2 samples), depth 8,
    NEE + MIS, Russian roulette off; also with the reference's default RR on."""
    sb, cam, cfg = cornell_box(0)
    assert (cfg.width, cfg.height, cfg.spp, cfg.max_bounces) == (320, 180, 16, 8)
    assert cfg.flags & _abi.RM_FLAG_NO_RR
    if rr:
        cfg.flags &= ~_abi.RM_FLAG_NO_RR
    sc = oracle.with_reference_bvh(sb.pack())
    assert sc.n_tris == 36
    o = oracle.Oracle()
    o_rgb, o_hdr, o_st = o.render(sc, cam, cfg, 12345)
    backend.stats_reset()
    g_rgb, g_hdr = backend.render(sc, cam, cfg, 12345, hdr=True, use_nodes=False)
    st = backend.stats()
    npix = cfg.width * cfg.height
    assert st["kernel_chain"] == o_st["chain"] == 8
    assert np.array_equal(backend.debug_read(4, npix), o.debug_read(4, npix)), "RNG state / sample count differ"
    assert exact_fraction(g_hdr, o_hdr) == 1.0
    assert np.array_equal(g_rgb, o_rgb)
    assert st["path_samples"] == o_st["path_samples"] and st["rays"] == o_st["rays"]


@pytest.mark.parametrize("denoise", [False, True], ids=["raw", "denoised"])
def test_animated_history_matches_oracle(oracle, denoise):
    """Three frames of a small animated sequence with temporal ReSTIR (and the
    temporal denoiser) on moving geometry: the device world (refitted after
    the first frame) against the oracle on the host-built world of each frame,
    with its own history carried from frame to frame.  A context of its own,
    so that its commit count (the rebuild schedule) starts at zero."""
    import torch
    import raymotion_b200 as rb
    backend = rb.Backend(0)
    seq = AnimatedSequence(seed=2, n_spheres=14, subdiv=2, n_emitters=96, cloth_verts=24, frames=3, width=128,
                           height=72, spp=4, depth=6, moving=0.5)
    cfg = seq.cfg
    cfg.restir_candidates, cfg.restir_spatial, cfg.restir_radius = 8, 3, 10.0
    cfg.flags = _abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_ANIMATED_HISTORY | (0 if denoise else _abi.RM_FLAG_DENOISE_OFF)
    npix = cfg.width * cfg.height
    ids = [backend.model_create(m) for m in seq.models]
    backend.reset_history()
    o = oracle.Oracle()
    st0 = backend.stats()
    d_rgb = torch.empty(npix * 3, dtype=torch.uint8, device="cuda")
    d_hdr = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
    for f in range(seq.frames):
        cloth = seq.cloth(f)
        backend.model_update(ids[seq.CLOTH], cloth)
        insts = seq.instances(f)
        recs = objects.instance_records(insts)
        recs["model"] = np.asarray(ids, np.int32)[recs["model"]]
        backend.instances_commit(recs, rebuild_every=32)
        cam = seq.camera(f)
        backend.render_resident_async(cam, cfg, 500 + f, d_rgb.data_ptr(), d_hdr.data_ptr())
        backend.sync()
        models = list(seq.models)
        models[seq.CLOTH] = cloth
        world = oracle.with_reference_bvh(objects.world_builder(models, insts).pack())
        o_rgb, o_hdr, o_st = o.render(world, cam, cfg, 500 + f)
        assert o_st["chain"] == 2 and backend.stats()["kernel_chain"] == 2
        g = _frame_buffers(backend, npix)
        r = _frame_buffers(o, npix)
        _compare_band(g, r, cfg.width, 0, cfg.height, f"frame {f}")
        # from the second frame on, temporal reuse merges history: some merged
        # reservoirs then count more samples than the pixel and its neighbours hold
        m_own = int(r["r_init"]["M"].max()) * (1 + cfg.restir_spatial)
        assert (r["r_merged"]["M"] > m_own).any() == (f > 0), f
        g_hdr = d_hdr.cpu().numpy()
        if denoise:
            assert rel_close_fraction(g_hdr, o_hdr, 1e-4) >= 0.999, f
        else:
            assert exact_fraction(g_hdr, o_hdr) == 1.0, f
            assert np.array_equal(d_rgb.cpu().numpy(), o_rgb), f
    st = backend.stats()
    assert st["bvh_builds"] - st0["bvh_builds"] == 1 and st["bvh_refits"] - st0["bvh_refits"] == 2
    backend.close()
