"""The reference's known-answer tests (tests/test_metal.cpp, tests/test_alpha.cpp)
run on the CPU oracle: they pin its path-tracing restatement."""
import numpy as np

from raymotion_b200.scene import Camera, RenderConfig, SceneBuilder

from . import kat_scenes as K


def _render(oracle, o, scene, cam, cfg, seed):
    oracle.with_reference_bvh(scene)
    rgb, hdr, st = o.render(scene, cam, cfg, seed)
    return rgb


def test_metal_kats(oracle):
    o = oracle.Oracle()
    cam, cfg = K.metal_config()
    empty = SceneBuilder().pack()
    rgb, _, _ = o.render(empty, cam, cfg, 12345)
    assert not rgb.any(), "empty scene is not black"  # test_metal.cpp:28
    sc = K.metal_scene().pack()
    oracle.with_reference_bvh(sc, 2)
    a, _, _ = o.render(sc, cam, cfg, 12345)
    assert a.any(), "lit scene is black"  # :43
    b, _, _ = o.render(sc, cam, cfg, 12345)
    assert np.array_equal(a, b), "not deterministic"  # :44-46
    cfg.adapt_min = 16
    em = K.fullscreen_emitter()
    rgb = _render(oracle, o, em, cam, cfg, 98765)
    px = rgb.reshape(-1, 3)
    assert (px[:, 0] == 127).all() and (px[:, 1:] == 0).all()  # :48-52
    cfg = RenderConfig(width=16, height=16, spp=2048, adapt_min=0)
    cam.focal = cfg.width * .8660254
    for opacity in (0.0, 0.5, 1.0):
        em = K.fullscreen_emitter(alpha=opacity)
        rgb = _render(oracle, o, em, cam, cfg, 98765).reshape(-1, 3)
        if opacity == .5:
            assert abs(rgb[:, 0].astype(float).mean() - 85) < 3  # :59-63
        if opacity == 0:
            assert not rgb.any()
        if opacity == 1:
            assert rgb[0, 0] == 127
    cfg = RenderConfig(width=37, height=23, spp=9, adapt_min=0)
    for frame in range(6):  # :67-76 (34 frames on the GPU; the oracle checks the alternation)
        rgb = _render(oracle, o, K.fullscreen_emitter((frame % 2) * 100.0), cam, cfg, 12345).reshape(-1, 3)
        assert (rgb[:, 0] == (0 if frame % 2 else 127)).all() and not rgb[:, 1:].any()


def test_alpha_kats(oracle):
    o = oracle.Oracle()
    for opacity in (0.0, 0.5, 1.0):
        sc = K.alpha_pair(opacity).pack()
        cfg = RenderConfig(width=8, height=8, spp=4096, adapt_min=0)
        rgb = _render(oracle, o, sc, Camera(), cfg, 12345).reshape(-1, 3).astype(float)
        assert abs(rgb[:, 0].mean() - 255 * opacity / (1 + opacity)) < 3  # test_alpha.cpp:20
        assert abs(rgb[:, 1].mean() - 255 * (1 - opacity) / (2 - opacity)) < 3  # :21
    sc = K.alpha_layers().pack()
    rgb = _render(oracle, o, sc, Camera(), RenderConfig(width=1, height=1, spp=1), 12345)
    assert rgb[0] == 0 and rgb[1] == 127  # :23-29
    sb = SceneBuilder()
    K._surface(sb, 1, -1, (0, 0, 0))
    K._surface(sb, 2, 2, (0, 0, 0))
    t = sb.pack().tris
    assert t["alpha"][0] == 0 and t["alpha"][1] == 1  # :30-31
