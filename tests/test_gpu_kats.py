"""The reference's known-answer tests through the C ABI on the GPU:
tests/test_metal.cpp:19-76 and tests/test_alpha.cpp:13-31."""
import numpy as np
import pytest

import raymotion_b200 as rb
from raymotion_b200.scene import Camera, RenderConfig, SceneBuilder

from . import kat_scenes as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("use_nodes", [True, False], ids=["caller_bvh", "device_lbvh"])
def test_metal_kats_on_gpu(backend, oracle, use_nodes):
    cam, cfg = K.metal_config()
    empty = SceneBuilder().pack()
    assert not backend.render(empty, cam, cfg, 12345).any()
    sc = oracle.with_reference_bvh(K.metal_scene().pack(), 2)
    a = backend.render(sc, cam, cfg, 12345, use_nodes=use_nodes)
    assert a.any()
    b = backend.render(sc, cam, cfg, 12345, use_nodes=use_nodes)
    assert np.array_equal(a, b)
    cfg.adapt_min = 16
    em = oracle.with_reference_bvh(K.fullscreen_emitter())
    px = backend.render(em, cam, cfg, 98765, use_nodes=use_nodes).reshape(-1, 3)
    assert (px[:, 0] == 127).all() and not px[:, 1:].any()
    cfg = RenderConfig(width=16, height=16, spp=2048, adapt_min=0)
    cam.focal = cfg.width * .8660254
    for opacity in (0.0, 0.5, 1.0):
        em = oracle.with_reference_bvh(K.fullscreen_emitter(alpha=opacity))
        rgb = backend.render(em, cam, cfg, 98765, use_nodes=use_nodes).reshape(-1, 3)
        if opacity == .5:
            assert abs(rgb[:, 0].astype(float).mean() - 85) < 3
        if opacity == 0:
            assert not rgb.any()
        if opacity == 1:
            assert rgb[0, 0] == 127
    cfg = RenderConfig(width=37, height=23, spp=9, adapt_min=0)
    for frame in range(34):
        em = oracle.with_reference_bvh(K.fullscreen_emitter((frame % 2) * 100.0))
        rgb = backend.render(em, cam, cfg, 12345, use_nodes=use_nodes).reshape(-1, 3)
        assert (rgb[:, 0] == (0 if frame % 2 else 127)).all() and not rgb[:, 1:].any()


def test_alpha_kats_on_gpu(backend, oracle):
    for opacity in (0.0, 0.5, 1.0):
        sc = oracle.with_reference_bvh(K.alpha_pair(opacity).pack())
        cfg = RenderConfig(width=8, height=8, spp=4096, adapt_min=0)
        rgb = backend.render(sc, Camera(), cfg, 12345).reshape(-1, 3).astype(float)
        assert abs(rgb[:, 0].mean() - 255 * opacity / (1 + opacity)) < 3
        assert abs(rgb[:, 1].mean() - 255 * (1 - opacity) / (2 - opacity)) < 3
    sc = oracle.with_reference_bvh(K.alpha_layers().pack())
    rgb = backend.render(sc, Camera(), RenderConfig(width=1, height=1, spp=1), 12345)
    assert rgb[0] == 0 and rgb[1] == 127


def test_empty_caller_bvh_misses_everything(backend, oracle):
    """nodes present but empty = the reference's params.nodes == 0 (pathtrace.metal:121)."""
    cam, cfg = K.metal_config()
    cfg.spp = 8
    sc = K.metal_scene().pack()
    sc.nodes = np.zeros(0, dtype=rb._abi.BVH_NODE_DTYPE)
    sc.bvh_tri = np.zeros(0, np.int32)
    assert not backend.render(sc, cam, cfg, 1).any()


def test_render_image_metal_entry(backend, oracle):
    cam, cfg = K.metal_config()
    cfg.spp = 8
    ok, rgb, err = rb.render_image_metal(oracle.with_reference_bvh(K.metal_scene().pack(), 2), cam, cfg, 5)
    assert ok and err == "" and rgb.shape == (cfg.width * cfg.height * 3,) and rgb.any()
    ok, rgb, err = rb.render_image_metal(SceneBuilder().pack(), cam, RenderConfig(spp=0), 5)
    assert not ok and err == "Invalid Metal render dimensions or sample count"


def test_caller_bvh_validation(backend, oracle):
    sc = oracle.with_reference_bvh(K.metal_scene().pack(), 2)
    sc.nodes = sc.nodes.copy()
    sc.nodes["left"][0] = 0  # a cycle: child index not after its parent
    cam, cfg = K.metal_config()
    with pytest.raises(rb.RenderError) as ex:
        backend.render(sc, cam, cfg, 1)
    assert ex.value.code == rb._abi.RM_ERR_BVH


def test_preview_last_sends_the_frame_rendered(backend, oracle):
    """rmcuda_preview_last: the last frame's RGB8, tonemapped on the device from
    its final linear image, through the reference's preview framing."""
    import os

    from raymotion_b200.scenes import cornell_box
    sb, cam, cfg = cornell_box(0)
    sc = sb.pack()
    rgb = backend.render(sc, cam, cfg, 12345, use_nodes=False)
    import threading

    r, w = os.pipe()
    gr, gw = os.pipe()
    os.write(gw, b"g")
    chunks = []

    def drain():  # the frame is larger than a pipe's buffer
        while True:
            b = os.read(r, 1 << 20)
            if not b:
                break
            chunks.append(b)

    t = threading.Thread(target=drain)
    t.start()
    assert backend.preview_last(w, 3, gr)
    os.close(w)
    t.join(timeout=30)
    head, body = b"".join(chunks).split(b"\n", 1)
    assert head == f"RAY1 {cfg.width} {cfg.height} 3 {cfg.width * cfg.height * 3}".encode()
    assert body == rgb.tobytes()
    for fd in (r, gr, gw):
        os.close(fd)
