"""Convergence of the CUDA plain path tracer to the oracle's FP64 render.

The FP64 instantiation of the oracle (one RNG stream per (pixel, sample),
1024 spp) is the converged reference R.  The CUDA path renders K frames of
N spp with independent seeds; with the clamp off the estimator is unbiased,
so over all pixel channels with R > 0:
  * the normalised sum T = sum(m - R) / sqrt(sum(var(m) + var(R))) of the
    K-frame means m is a standard normal (|T| < 5 here), with var(m) from the
    K frames and var(R) from the same per-sample variance at 1024 spp;
  * relMSE = mean((I - R)^2 / (R^2 + 0.01)) falls about K-fold from one frame
    to the mean of K frames (noise, not bias, dominates).
"""
import numpy as np
import pytest

from raymotion_b200 import _abi
from raymotion_b200.scenes import icosphere_field

pytestmark = pytest.mark.gpu


def relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 0.01)))


def test_plain_path_converges_to_the_fp64_oracle(backend, oracle):
    sb, cam, cfg = icosphere_field(seed=5, n_spheres=12, subdiv=2, n_emitters=64, width=80, height=48, spp=16,
                                   depth=5)
    sc = oracle.with_reference_bvh(sb.pack())
    cfg.clamp = 0.0
    cfg.adapt_min = 0
    cfg.flags = _abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_RESTIR_OFF | _abi.RM_FLAG_DENOISE_OFF
    ref_spp = 1024
    rcfg = type(cfg)(**{**cfg.__dict__, "spp": ref_spp})
    ref = oracle.render_f64(sc, cam, rcfg, 4242).reshape(-1, 3)
    K = 16
    frames = []
    for k in range(K):
        _, hdr = backend.render(sc, cam, cfg, 1000 + k, hdr=True, use_nodes=False)
        frames.append(hdr.reshape(-1, 3).astype(np.float64))
    frames = np.stack(frames)
    m = frames.mean(0)
    var_frame = frames.var(0, ddof=1)
    var_m = var_frame / K
    var_ref = var_frame * cfg.spp / ref_spp
    live = ref > 0
    assert live.mean() > 0.3
    T = (m - ref)[live].sum() / np.sqrt((var_m + var_ref)[live].sum())
    assert abs(T) < 5.0, T
    single = np.mean([relmse(f, ref) for f in frames])
    assert relmse(m, ref) < single / 6, (relmse(m, ref), single)
