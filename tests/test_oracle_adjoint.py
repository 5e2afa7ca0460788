"""The oracle's frozen-path evaluator, the finite-difference side of the adjoint check (CPU).

orc_render_frozen replays the fp32 plain frame and evaluates each sample's
material-dependent factors in double at given parameters.  At the scene's own
parameters it must reproduce the fp32 frame (in double); the emission enters
every path contribution exactly once, so with the clamp off the frame is
linear in the lights' emission; and it must be smooth enough for central
differences (second differences small next to first differences).
"""
import numpy as np
import pytest

from raymotion_b200 import _abi
from raymotion_b200.scene import with_materials
from raymotion_b200.scenes import inverse_scene


@pytest.fixture(scope="module")
def small(oracle):
    d = inverse_scene(seed=7, n_spheres=10, subdiv=2, ground=20, patches=(3, 3), n_emitters=3, n_dielectric=3,
                      width=40, height=32, spp=4, depth=6)
    oracle.with_reference_bvh(d["scene"])
    return d


def ris_config(cfg, candidates=8):
    """The plain chain with RIS NEE over `candidates` lights per vertex."""
    return type(cfg)(**{**cfg.__dict__, "restir_candidates": candidates, "restir_spatial": 0,
                        "flags": cfg.flags & ~_abi.RM_FLAG_RESTIR_OFF})


@pytest.mark.parametrize("nee", ["single", "ris8"])
def test_frozen_at_scene_parameters_is_the_fp32_frame(oracle, small, nee):
    sc, cam, cfg = small["scene"], small["camera"], small["config"]
    if nee == "ris8":
        cfg = ris_config(cfg)
    _, hdr, _ = oracle.Oracle().render(sc, cam, cfg, 99)
    fro = oracle.render_frozen(sc, cam, cfg, 99, small["tri_material"], small["params"].astype(np.float64))
    hdr = hdr.reshape(-1, 3).astype(np.float64)
    assert hdr.max() > 0.05
    # the double evaluation differs from fp32 by rounding, most near the peak
    # of smooth GGX lobes (alpha2 down to 6e-6), where 1 - cos_h^2 cancels
    rel = np.abs(fro - hdr) / (np.abs(hdr) + 1e-7)
    assert np.median(rel) < 1e-6
    assert rel.max() < 5e-4


@pytest.mark.parametrize("nee", ["single", "ris8"])
def test_frozen_frame_is_linear_in_emission(oracle, small, nee):
    """RIS NEE holds its selection and resampling weight, so its light sample
    is Le f k with k fixed: still linear in the emission."""
    sc, cam, cfg = small["scene"], small["camera"], small["config"]
    if nee == "ris8":
        cfg = ris_config(cfg)
    cfg.clamp = 0.0
    prm = small["params"].astype(np.float64)
    a = oracle.render_frozen(sc, cam, cfg, 5, small["tri_material"], prm)
    prm2 = prm.copy()
    prm2[:, 4:7] *= 2.0
    b = oracle.render_frozen(sc, cam, cfg, 5, small["tri_material"], prm2)
    assert np.allclose(b, 2.0 * a, rtol=1e-12, atol=1e-15)
    cfg.clamp = 16.0


@pytest.mark.parametrize("col", [0, 3, 4, 7], ids=["albedo_r", "rough", "emission_r", "ior"])
def test_frozen_frame_is_smooth_for_central_differences(oracle, small, col):
    sc, cam, cfg = small["scene"], small["camera"], small["config"]
    prm = small["params"].astype(np.float64)
    rows = np.nonzero(small["mask"][:, col])[0][:3]
    h = 1e-3
    for m in rows:
        vals = []
        for k in (-2, -1, 1, 2):
            q = prm.copy()
            q[m, col] += k * h
            vals.append(oracle.render_frozen(sc, cam, cfg, 11, small["tri_material"], q).sum())
        # central differences at h and 2h: their truncation errors (h^2 f'''/6
        # and four times that) differ by three times the error of the h estimate
        d1 = (vals[2] - vals[1]) / (2 * h)
        d2 = (vals[3] - vals[0]) / (4 * h)
        assert abs(d1 - d2) <= 3e-4 * abs(d1) + 1e-9, (m, col, d1, d2)


def test_with_materials_matches_builder_light_table(small):
    d = small
    again = with_materials(d["scene"], d["tri_material"], d["params"])
    assert np.array_equal(again.light_cdf, d["scene"].light_cdf)
    assert again.light_total == d["scene"].light_total
    for name in ("ar", "rough", "er", "ior"):
        assert np.array_equal(again.tris[name], d["scene"].tris[name])


def restir_config(cfg, spp=4, denoise=False):
    """The ReSTIR chain (first frame) on the same scene."""
    flags = cfg.flags & ~_abi.RM_FLAG_RESTIR_OFF & ~_abi.RM_FLAG_DENOISE_OFF
    return type(cfg)(**{**cfg.__dict__, "spp": spp, "restir_candidates": 4, "restir_spatial": 2,
                        "restir_radius": 6.0, "flags": flags | (0 if denoise else _abi.RM_FLAG_DENOISE_OFF)})


@pytest.mark.parametrize("denoise", [False, True], ids=["raw", "denoised"])
def test_frozen_restir_frame_at_scene_parameters_is_the_fp32_frame(oracle, small, denoise):
    sc, cam = small["scene"], small["camera"]
    cfg = restir_config(small["config"], denoise=denoise)
    o = oracle.Oracle()
    _, hdr, st = o.render(sc, cam, cfg, 77)
    assert st["chain"] == 2
    fro = oracle.render_frozen_restir(sc, cam, cfg, 77, small["tri_material"], small["params"].astype(np.float64))
    hdr = hdr.reshape(-1, 3).astype(np.float64)
    assert hdr.max() > 0.05
    rel = np.abs(fro - hdr) / (np.abs(hdr) + 1e-7)
    if not denoise:
        assert np.median(rel) < 1e-6
        assert rel.max() < 5e-4
    else:
        # the a-trous weights in double against the fp32 pass: luma differences
        # in the exponents carry fp32 rounding (as the CUDA filter's 1e-4)
        assert np.median(rel) < 1e-5
        assert np.quantile(rel, 0.999) < 5e-4 and rel.max() < 2e-3


def test_frozen_restir_frame_is_linear_in_emission(oracle, small):
    sc, cam = small["scene"], small["camera"]
    cfg = restir_config(small["config"])
    cfg.clamp = 0.0
    prm = small["params"].astype(np.float64)
    a = oracle.render_frozen_restir(sc, cam, cfg, 5, small["tri_material"], prm)
    prm2 = prm.copy()
    prm2[:, 4:7] *= 2.0
    b = oracle.render_frozen_restir(sc, cam, cfg, 5, small["tri_material"], prm2)
    assert np.allclose(b, 2.0 * a, rtol=1e-12, atol=1e-15)
    assert np.abs(a).max() > 0


@pytest.mark.parametrize("denoise", [False, True], ids=["raw", "denoised"])
def test_frozen_restir_second_frame_is_the_fp32_frame(oracle, small, denoise):
    """A frame with temporal history: the frozen evaluation renders the first
    frame in fp32 for its history and reproduces the oracle's second frame."""
    sc, cam = small["scene"], small["camera"]
    cfg = restir_config(small["config"], denoise=denoise)
    o = oracle.Oracle()
    o.render(sc, cam, cfg, 90)
    _, hdr, st = o.render(sc, cam, cfg, 91)
    assert st["chain"] == 2
    fro = oracle.render_frozen_restir(sc, cam, cfg, 91, small["tri_material"], small["params"].astype(np.float64),
                                      prev=(cam, 90))
    first = oracle.render_frozen_restir(sc, cam, cfg, 91, small["tri_material"], small["params"].astype(np.float64))
    hdr = hdr.reshape(-1, 3).astype(np.float64)
    rel = np.abs(fro - hdr) / (np.abs(hdr) + 1e-7)
    assert np.median(rel) < 1e-5
    assert np.quantile(rel, 0.999) < 5e-4 and rel.max() < 2e-3
    assert not np.allclose(first, hdr, rtol=1e-3)  # the history mattered
