"""Path-replay adjoint (rmcuda_backward) against FP64 central differences and
against a 16,384-spp reference gradient (GPU).

The loss is L = mean((I - T)^2) over a W x H x 3 radiance image I of the
plain frame, T a fixed target.  The adjoint's dL/dparams (given dL/dI at the
current parameters) is compared with central differences of L (h = 1e-3,
Richardson-extrapolated with h/2) evaluated by the oracle's frozen-path
renderer in double: the same paths as
the fp32 frame (sampling held at the current parameters), material factors at
the perturbed parameters.  For each parameter kind (albedo r/g/b, roughness,
emission r/g/b, ior) the check takes the materials with the largest gradients
and one more; gradients above 1 % of the kind's largest must agree within
1e-3 relative, the rest within 1e-5 of that largest.

The torch.autograd.Function below exists only in this test harness: it wraps
rmcuda_render_scene_async / rmcuda_backward so that torch's optimiser can
drive them.
"""
import numpy as np
import pytest

from raymotion_b200 import RenderError, _abi
from raymotion_b200.scene import RenderConfig, with_materials
from raymotion_b200.scenes import inverse_scene

pytestmark = pytest.mark.gpu

H = 1e-3


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _scene(oracle, spp, depth=6):
    # 8 of the 10 spheres dielectric, so that several are in view
    d = inverse_scene(seed=7, n_spheres=10, subdiv=2, ground=20, patches=(3, 3), n_emitters=3, n_dielectric=8,
                      width=48, height=40, spp=spp, depth=depth)
    oracle.with_reference_bvh(d["scene"])
    return d


def _set(backend, h, d, params):
    s = with_materials(d["scene"], d["tri_material"], params)
    backend.scene_set_materials(h, params, d["tri_material"], s.light_cdf, s.light_total)


def _render(backend, h, d, seed):
    torch = _torch()
    cfg = d["config"]
    img = torch.empty(cfg.width * cfg.height * 3, dtype=torch.float32, device="cuda")
    backend.render_scene_async(h, d["camera"], cfg, seed, None, img.data_ptr())
    backend.sync()
    return img


def _grad(backend, h, d, seed, dl):
    torch = _torch()
    g = torch.zeros(d["params"].size, dtype=torch.float32, device="cuda")
    backend.backward(h, d["camera"], d["config"], seed, dl.data_ptr(), g.data_ptr())
    backend.sync()
    return g.cpu().numpy().reshape(-1, 8)


def central_difference(loss, prm, m, col, h0=H):
    """Central differences at H and H/2, Richardson-extrapolated: the plain
    H-difference carries an H^2 error of up to a few percent on the peaks of
    glossy lobes and near a dielectric's critical angle, where the frame's
    third derivative is large."""
    def d(h):
        qp, qm = prm.copy(), prm.copy()
        qp[m, col] += h
        qm[m, col] -= h
        return (loss(qp) - loss(qm)) / (2 * h)
    return (4.0 * d(h0 / 2) - d(h0)) / 3.0


@pytest.mark.parametrize("spp,candidates", [(4, 1), (8, 1), (4, 8)], ids=["one_lane", "eight_lanes", "ris_nee"])
def test_adjoint_matches_fp64_central_differences(backend, oracle, spp, candidates):
    """ris_nee: the plain chain with RIS over 8 light candidates per vertex;
    the selection and its resampling weight are held on both sides."""
    torch = _torch()
    d = _scene(oracle, spp)
    if candidates > 1:
        c = d["config"]
        d["config"] = type(c)(**{**c.__dict__, "restir_candidates": candidates, "restir_spatial": 0,
                                 "flags": c.flags & ~_abi.RM_FLAG_RESTIR_OFF})
    seed = 2024
    sc, cam, cfg, tm = d["scene"], d["camera"], d["config"], d["tri_material"]
    prm = d["params"].astype(np.float64)
    h = backend.scene_create(sc)
    try:
        _set(backend, h, d, d["params"])
        img = _render(backend, h, d, seed)
        T = (img.cpu().numpy() * np.float32(0.75) + np.float32(0.01)).reshape(-1, 3).astype(np.float64)
        # dL/dI of the loss on the FP64 image (the fp32 frame differs from it by
        # rounding, up to ~3e-4 near the peaks of smooth GGX lobes)
        i64 = oracle.render_frozen(sc, cam, cfg, seed, tm, prm)
        dl = torch.from_numpy(((2.0 / i64.size) * (i64 - T)).astype(np.float32).ravel()).cuda()
        g = _grad(backend, h, d, seed, dl)
    finally:
        backend.scene_destroy(h)

    def loss(q):
        return np.mean((oracle.render_frozen(sc, cam, cfg, seed, tm, q) - T) ** 2)

    rng = np.random.default_rng(0)
    checks = []
    for col in range(8):
        cand = np.nonzero(d["mask"][:, col])[0]
        top = cand[np.argsort(-np.abs(g[cand, col]))][:3]
        extra = rng.choice(cand, 1)
        for m in sorted(set(top.tolist()) | set(extra.tolist())):
            checks.append((m, col, central_difference(loss, prm, m, col), float(g[m, col])))
    significant = 0
    for col in range(8):
        rows = [c for c in checks if c[1] == col]
        big = max(abs(c[2]) for c in rows)
        assert big > 0, f"param {col}: no gradient"
        for (m, _, f, a) in rows:
            if abs(f) >= 1e-2 * big:
                significant += 1
                assert abs(a - f) <= 1e-3 * abs(f), f"material {m} param {col}: adjoint {a} vs FD {f}"
            else:
                assert abs(a - f) <= 1e-5 * big, f"material {m} param {col}: adjoint {a} vs FD {f}"
    assert significant >= 16


def test_backward_rejects_what_it_does_not_differentiate(backend, oracle):
    torch = _torch()
    d = _scene(oracle, 4)
    h = backend.scene_create(d["scene"])
    try:
        dl = torch.zeros(d["config"].width * d["config"].height * 3, device="cuda")
        g = torch.zeros(d["params"].size, device="cuda")
        with pytest.raises(RenderError, match="no materials"):
            backend.backward(h, d["camera"], d["config"], 1, dl.data_ptr(), g.data_ptr())
        _set(backend, h, d, d["params"])
        adaptive = d["config"]
        adaptive.flags &= ~0x2  # RM_FLAG_NOADAPT off
        adaptive.adapt_min = 16
        with pytest.raises(RenderError, match="fixed sample count"):
            backend.backward(h, d["camera"], adaptive, 1, dl.data_ptr(), g.data_ptr())
    finally:
        backend.scene_destroy(h)


def _render_function():
    torch = _torch()

    class RenderMaterials(torch.autograd.Function):
        """image = plain frame of the scene object with material parameters `params` (n x 8)."""

        @staticmethod
        def forward(ctx, params, backend, h, d, seed, adjoint_seed):
            p = params.detach().cpu().numpy().astype(np.float32)
            _set(backend, h, d, p)
            img = _render(backend, h, d, seed)
            ctx.backend, ctx.h, ctx.d, ctx.seed = backend, h, d, adjoint_seed
            return img

        @staticmethod
        def backward(ctx, grad_img):
            # adjoint_seed == seed differentiates this frame's own paths; another
            # seed gives an unbiased gradient of the expected loss for a
            # stochastic fit (the same paths bias it towards lower variance)
            g = _grad(ctx.backend, ctx.h, ctx.d, ctx.seed, grad_img.contiguous())
            return torch.from_numpy(g).to(grad_img.device), None, None, None, None, None

    return RenderMaterials


def test_autograd_function_and_a_short_fit(backend, oracle):
    """Fit the ground patches' albedo back from a +-30 % start.  Russian
    roulette off and one seed for the target and every step: the paths then
    do not depend on albedo, so the loss is a smooth function of it with its
    minimum, zero, at the true values."""
    torch = _torch()
    Fn = _render_function()
    d = _scene(oracle, 4)
    d["config"].flags |= 0x40  # RM_FLAG_NO_RR
    lo = torch.tensor([0.05, 0.05, 0.05, 0.05, 0.0, 0.0, 0.0, 1.3], device="cuda")
    hi = torch.tensor([0.95, 0.95, 0.95, 1.0, 20.0, 20.0, 20.0, 1.7], device="cuda")
    fit = np.zeros_like(d["mask"])
    fit[10:19, 0:3] = True  # the ground patches, in view everywhere
    mask = torch.from_numpy(fit & d["mask"]).cuda()
    true = torch.from_numpy(d["params"]).cuda()
    seed = 99
    h = backend.scene_create(d["scene"])
    try:
        target = Fn.apply(true, backend, h, d, seed, seed).detach()
        gen = torch.Generator(device="cuda").manual_seed(3)
        noise = (torch.rand(true.shape, device="cuda", generator=gen) * 2 - 1) * 0.3
        start = torch.where(mask, torch.clamp(true * (1 + noise), lo, hi), true)
        u = ((start - lo) / (hi - lo)).clone().requires_grad_(True)
        opt = torch.optim.Adam([u], lr=1e-2)
        # the gradient through the Function equals a direct rmcuda_backward call
        params = torch.where(mask, lo + (hi - lo) * u, true)
        img = Fn.apply(params, backend, h, d, seed, seed)
        loss = ((img - target) ** 2).mean()
        loss.backward()
        dl = (2.0 / img.numel()) * (img - target)
        direct = torch.from_numpy(_grad(backend, h, d, seed, dl.detach())).cuda()
        expect = torch.where(mask, direct * (hi - lo), torch.zeros_like(direct))
        assert torch.allclose(u.grad, expect, rtol=1e-4, atol=1e-9)
        err0 = ((params - true).abs() / (hi - lo))[mask].mean().item()
        loss0 = loss.item()
        for it in range(100):
            opt.zero_grad()
            params = torch.where(mask, lo + (hi - lo) * u.clamp(0, 1), true)
            img = Fn.apply(params, backend, h, d, seed, seed)
            loss = ((img - target) ** 2).mean()
            loss.backward()
            opt.step()
        params = torch.where(mask, lo + (hi - lo) * u.detach().clamp(0, 1), true)
        err1 = ((params - true).abs() / (hi - lo))[mask].mean().item()
        assert loss.item() < 0.05 * loss0, (loss0, loss.item())
        assert err1 < 0.5 * err0, (err0, err1)
    finally:
        backend.scene_destroy(h)




KINDS = {"albedo": [0, 1, 2], "roughness": [3], "emission": [4, 5, 6], "ior": [7]}


def test_gradients_converge_to_a_high_spp_reference_gradient(backend, oracle):
    """The adjoint's gradient of a linear loss L = sum(w * I) (fixed weights)
    at 4 spp (one lane per pixel), 64 and 1024 spp (32 lanes) against a
    16,384-spp reference gradient G of the same adjoint (its own seed).  Per
    parameter kind, the relative error e = |g - G| / |G| over the fitted
    parameters is Monte Carlo noise about G: for albedo, roughness and
    emission its RMS over 12 seeds falls about 4x per 16x spp (the checks ask
    for 2x; a biased lane kernel or sample weighting would leave a floor), is
    small at 1024 spp, and the mean of 16 one-lane frames at 4 spp (64 spp in
    all) is as close to G as a 64-spp frame.  The IOR gradient's estimator is
    heavy-tailed (the refraction's derivative grows without bound towards the
    critical angle), so its RMS does not fall steadily; its median error
    must still fall.  Measured on a B200: RMS e at 4 / 64 / 1024 spp albedo
    0.014 / 0.0037 / 0.0010, roughness 0.57 / 0.12 / 0.031, emission 0.055 /
    0.012 / 0.0038; IOR median 0.45 / 0.16 / 0.09."""
    torch = _torch()
    d = _scene(oracle, 4)
    base = d["config"]
    npix = base.width * base.height
    w = np.random.default_rng(11).uniform(0.5, 1.5, npix * 3).astype(np.float32) / np.float32(npix * 3)
    dl = torch.from_numpy(w).cuda()
    mask = d["mask"]

    def grad(spp, seed):
        cfg = type(base)(**{**base.__dict__, "spp": spp})
        g = torch.zeros(d["params"].size, dtype=torch.float32, device="cuda")
        backend.backward(h, d["camera"], cfg, seed, dl.data_ptr(), g.data_ptr())
        backend.sync()
        return g.cpu().numpy().reshape(-1, 8).astype(np.float64)

    h = backend.scene_create(d["scene"])
    try:
        _set(backend, h, d, d["params"])
        G = grad(16384, 777)
        runs = {spp: [grad(spp, 1000 * spp + k) for k in range(12)] for spp in (4, 64, 1024)}
        mean4 = np.mean([grad(4, 50000 + k) for k in range(16)], axis=0)
    finally:
        backend.scene_destroy(h)

    report = {}
    for kind, cols in KINDS.items():
        m = mask[:, cols]
        ref = np.linalg.norm(G[:, cols][m])
        assert ref > 0, kind
        errs = {spp: np.array([np.linalg.norm((g[:, cols] - G[:, cols])[m]) / ref for g in gs])
                for spp, gs in runs.items()}
        report[kind] = dict(rms={k: round(float(np.sqrt(np.mean(e ** 2))), 5) for k, e in errs.items()},
                            median={k: round(float(np.median(e)), 5) for k, e in errs.items()},
                            mean4=round(float(np.linalg.norm((mean4[:, cols] - G[:, cols])[m]) / ref), 5))
    for kind, top in (("albedo", 0.005), ("roughness", 0.1), ("emission", 0.02)):
        r = report[kind]
        assert r["rms"][4] > 2.0 * r["rms"][64] and r["rms"][64] > 2.0 * r["rms"][1024], report
        assert r["rms"][1024] < top, report
        assert r["mean4"] < 3.0 * r["rms"][64], report
    assert report["ior"]["median"][1024] < 0.5 * report["ior"]["median"][4], report


@pytest.mark.parametrize("denoise,second", [(False, False), (True, False), (True, True)],
                         ids=["raw", "denoised", "denoised_with_history"])
def test_restir_frame_adjoint_matches_fp64_central_differences(backend, oracle, denoise, second):
    """The ReSTIR chain (K3 4 candidates with visibility, K4 2 neighbours, K5,
    and the denoiser when on; first frame): the adjoint takes the loss
    gradient back through the denoiser (G-buffer held) and replays K5 from the
    checkpoint the frame left (its G-buffer and merged reservoirs); the oracle
    runs K3/K4 in fp32 and evaluates K5 frozen and the denoiser in double.
    with_history: the frame is the second of a history (temporal reservoir
    reuse and the temporal blend; the oracle renders the first in fp32).
    Same acceptance as the plain frame's check."""
    torch = _torch()
    d = _scene(oracle, 4)
    c = d["config"]
    flags = c.flags & ~_abi.RM_FLAG_RESTIR_OFF & ~_abi.RM_FLAG_DENOISE_OFF
    cfg = type(c)(**{**c.__dict__, "restir_candidates": 4, "restir_spatial": 2, "restir_radius": 6.0,
                     "flags": flags | (0 if denoise else _abi.RM_FLAG_DENOISE_OFF)})
    d["config"] = cfg
    seed = 515
    sc, cam, tm = d["scene"], d["camera"], d["tri_material"]
    prm = d["params"].astype(np.float64)
    h = backend.scene_create(sc)
    try:
        _set(backend, h, d, d["params"])
        backend.reset_history()
        prev = None
        if second:
            _render(backend, h, d, seed - 7)
            prev = (cam, seed - 7)
        img = _render(backend, h, d, seed)  # the frame whose G-buffer and reservoirs are the checkpoint
        assert backend.stats()["kernel_chain"] == 2
        T = (img.cpu().numpy() * np.float32(0.75) + np.float32(0.01)).reshape(-1, 3).astype(np.float64)
        i64 = oracle.render_frozen_restir(sc, cam, cfg, seed, tm, prm, prev=prev)
        assert np.allclose(i64, img.cpu().numpy().reshape(-1, 3), rtol=2e-3, atol=1e-5)
        dl = torch.from_numpy(((2.0 / i64.size) * (i64 - T)).astype(np.float32).ravel()).cuda()
        g = _grad(backend, h, d, seed, dl)
        # the checkpoint must be this frame's, with the materials it was rendered with
        with pytest.raises(RenderError, match="replays the last frame"):
            _grad(backend, h, d, seed + 1, dl)
        if not second:
            _set(backend, h, d, d["params"])
            with pytest.raises(RenderError, match="replays the last frame"):
                _grad(backend, h, d, seed, dl)
    finally:
        backend.scene_destroy(h)

    def loss(q):
        return np.mean((oracle.render_frozen_restir(sc, cam, cfg, seed, tm, q, prev=prev) - T) ** 2)

    rng = np.random.default_rng(1)
    checks = []
    for col in range(8):
        cand = np.nonzero(d["mask"][:, col])[0]
        top = cand[np.argsort(-np.abs(g[cand, col]))][:3]
        extra = rng.choice(cand, 1)
        for m in sorted(set(top.tolist()) | set(extra.tolist())):
            checks.append((m, col, central_difference(loss, prm, m, col), float(g[m, col])))
    significant = 0
    for col in range(8):
        rows = [ch for ch in checks if ch[1] == col]
        big = max(abs(ch[2]) for ch in rows)
        assert big > 0, f"param {col}: no gradient"
        for (m, _, f, a) in rows:
            if abs(f) >= 1e-2 * big:
                significant += 1
                assert abs(a - f) <= 1e-3 * abs(f), f"material {m} param {col}: adjoint {a} vs FD {f}"
            else:
                assert abs(a - f) <= 1e-5 * big, f"material {m} param {col}: adjoint {a} vs FD {f}"
    assert significant >= 12


def test_adjoint_on_a_textured_scene_matches_fp64_central_differences(backend, oracle):
    """The known-answer scene with its 2x2 texture on walls, metal and both
    dielectrics, one material per quad: the albedo derivative carries the
    texel (the G-buffer and BSDF albedo are albedo x texel).  Plain chain,
    single-candidate NEE; every material's albedo and roughness, the light's
    emission and the dielectrics' IOR against FP64 central differences with a
    step of 1e-5: the loss's third derivative in the rough dielectric quad's
    roughness is large enough that steps of 1e-3 and 5e-4 (Richardson) are 7 %
    off, while the differences at 1e-4 ... 1e-6 agree to seven digits."""
    from raymotion_b200.scenes import PLAIN_FLAGS

    from . import kat_scenes as K
    torch = _torch()
    cam, _ = K.metal_config()
    cfg = RenderConfig(width=96, height=64, spp=4, max_bounces=6, adapt_min=0,
                       flags=PLAIN_FLAGS | _abi.RM_FLAG_NOADAPT)
    sc = K.metal_scene().pack()
    oracle.with_reference_bvh(sc, 2)
    t = sc.tris
    tm = (np.arange(len(t)) // 2).astype(np.int32)
    n_mat = int(tm.max()) + 1
    params = np.stack([t[k][::2] for k in ("ar", "ag", "ab", "rough", "er", "eg", "eb", "ior")], 1).astype(np.float32)
    mask = np.zeros((n_mat, 8), bool)
    mask[:, 0:4] = True
    mask[params[:, 4:7].max(1) > 0, 4:7] = True
    mask[params[:, 7] > 1.0001, 7] = True
    d = dict(scene=sc, tri_material=tm, params=params, camera=cam, config=cfg)
    seed = 808
    prm = params.astype(np.float64)
    h = backend.scene_create(sc)
    try:
        _set(backend, h, d, params)
        img = _render(backend, h, d, seed)
        T = (img.cpu().numpy() * np.float32(0.75) + np.float32(0.01)).reshape(-1, 3).astype(np.float64)
        i64 = oracle.render_frozen(sc, cam, cfg, seed, tm, prm)
        dl = torch.from_numpy(((2.0 / i64.size) * (i64 - T)).astype(np.float32).ravel()).cuda()
        g = _grad(backend, h, d, seed, dl)
    finally:
        backend.scene_destroy(h)

    def loss(q):
        return np.mean((oracle.render_frozen(sc, cam, cfg, seed, tm, q) - T) ** 2)

    fd = {(m, col): central_difference(loss, prm, m, col, 1e-5) for m, col in zip(*np.nonzero(mask))}
    significant = 0
    for cols in ([0, 1, 2], [3], [4, 5, 6], [7]):
        rows = [(k, f) for k, f in fd.items() if k[1] in cols]
        big = max(abs(f) for _, f in rows)
        assert big > 0, cols
        for (m, col), f in rows:
            a = float(g[m, col])
            if abs(f) >= 1e-2 * big:
                significant += 1
                assert abs(a - f) <= 1e-3 * abs(f), f"material {m} param {col}: adjoint {a} vs FD {f}"
            else:
                assert abs(a - f) <= 1e-5 * big, f"material {m} param {col}: adjoint {a} vs FD {f}"
    assert significant >= 12
