"""Batched rendering (rmcuda_render_batch) against the one-image plain path (GPU).

Every image of a batch must equal, bit for bit, what the single-frame policy
renders for it alone (rmcuda_render_scene_async, itself pinned to the CPU
oracle by test_gpu_parity.py): radiance, RGB8, and per pixel the XOR of the
lanes' final RNG states and the number of samples taken.  The batches mix the
lane kernels' shapes (1, 8 and 32 lanes, partial last rounds, adaptive early
exits), ragged tiles, a depth-0 image, and a partially transparent textured
scene whose extension and shadow rays draw random numbers.
"""
import numpy as np
import pytest

from raymotion_b200 import BatchItem, RenderError, _abi
from raymotion_b200.scene import RenderConfig
from raymotion_b200.scenes import cornell_box, sized_field

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _cfg(base, **kw):
    c = RenderConfig(**{f: getattr(base, f) for f in base.__dataclass_fields__})
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _mixed_images():
    """(packed scene, camera, config, seed, lanes) of the test batch."""
    from . import kat_scenes as K
    out = []
    sb, cam, cfg = cornell_box(0)
    cfg.flags = _abi.RM_FLAG_NO_ENV
    corn = sb.pack()
    out.append((corn, cam, _cfg(cfg, width=97, height=61, spp=16, adapt_min=16), 12345, 8))
    out.append((corn, cam, _cfg(cfg, width=33, height=17, spp=40, adapt_min=0), 99, 32))
    out.append((corn, cam, _cfg(cfg, width=40, height=30, spp=3, adapt_min=16), 5, 1))
    out.append((corn, cam, _cfg(cfg, width=24, height=9, spp=8, max_bounces=0), 6, 8))
    sb, cam, cfg = sized_field(seed=11, n_tris=30000, width=120, height=70, spp=20, depth=9)
    field = sb.pack()
    out.append((field, cam, _cfg(cfg, adapt_min=16, adapt_step=8), 777, 8))
    out.append((field, cam, _cfg(cfg, width=64, height=36, spp=4), 778, 1))
    sb, cam, cfg = sized_field(seed=12, n_tris=3000, width=80, height=45, spp=64, depth=12)
    out.append((sb.pack(), cam, cfg, 31337, 8))
    cam, cfg = K.metal_config()
    cfg = _cfg(cfg, spp=24, flags=_abi.RM_FLAG_NO_ENV | _abi.RM_FLAG_NOMIS | _abi.RM_FLAG_NO_RR |
               _abi.RM_FLAG_RESTIR_OFF)
    sc = K.metal_scene().pack()
    sc.tris["alpha"][::3] = np.float32(0.6)
    out.append((sc, cam, cfg, 4242, 8))
    return out


@pytest.fixture(scope="module")
def batch_case(backend):
    torch = _torch()
    images = _mixed_images()
    handles = {}
    refs = []
    for sc, cam, cfg, seed, lanes in images:
        if id(sc) not in handles:
            handles[id(sc)] = backend.scene_create(sc)
        h = handles[id(sc)]
        npix = cfg.width * cfg.height
        rgb = torch.empty(npix * 3, dtype=torch.uint8, device="cuda")
        hdr = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
        backend.stats_reset()
        backend.render_scene_async(h, cam, cfg, seed, rgb.data_ptr(), hdr.data_ptr())
        backend.sync()
        st = backend.stats()
        assert st["kernel_chain"] == lanes
        refs.append(dict(rgb=rgb.cpu().numpy(), hdr=hdr.cpu().numpy(), aux=backend.debug_read(4, npix),
                         samples=st["path_samples"]))
    yield images, handles, refs
    for h in handles.values():
        backend.scene_destroy(h)


def _render_batch(backend, images, handles):
    torch = _torch()
    outs, items = [], []
    for sc, cam, cfg, seed, _ in images:
        npix = cfg.width * cfg.height
        o = dict(rgb=torch.full((npix * 3,), 7, dtype=torch.uint8, device="cuda"),
                 hdr=torch.full((npix * 3,), -1.0, dtype=torch.float32, device="cuda"),
                 aux=torch.zeros(npix * 2, dtype=torch.int32, device="cuda"))
        outs.append(o)
        items.append(BatchItem(handles[id(sc)], cam, cfg, seed, o["rgb"].data_ptr(), o["hdr"].data_ptr(),
                               o["aux"].data_ptr()))
    backend.stats_reset()
    backend.render_batch(items)
    st = backend.stats()
    return [{k: v.cpu().numpy() for k, v in o.items()} for o in outs], st, (items, outs)


TUNINGS = [
    dict(pool_chunks=65536, tile_shape=0, grid_scale=1, graph_waves=8, bvh_width=2),
    dict(pool_chunks=5, tile_shape=1, grid_scale=1, graph_waves=2, bvh_width=2),
    dict(pool_chunks=37, tile_shape=0, grid_scale=2, graph_waves=0, bvh_width=2),
    dict(pool_chunks=65536, tile_shape=1, grid_scale=1, graph_waves=8, bvh_width=8),
]


@pytest.mark.parametrize("tuning", TUNINGS, ids=["default", "tiny_pool_graph2", "small_pool_nograph", "wide_bvh"])
def test_batch_equals_single_image_renders(backend, batch_case, tuning):
    images, handles, refs = batch_case
    backend.set_batch_tuning(**tuning)
    try:
        outs, st, _ = _render_batch(backend, images, handles)
    finally:
        backend.set_batch_tuning(**TUNINGS[0])
    for k, (o, r) in enumerate(zip(outs, refs)):
        assert np.array_equal(o["aux"].view(np.uint32), r["aux"]), f"image {k}: RNG state / sample count differ"
        assert np.array_equal(o["hdr"].view(np.uint32), r["hdr"].view(np.uint32)), f"image {k}: radiance differs"
        assert np.array_equal(o["rgb"], r["rgb"]), f"image {k}: RGB8 differs"
    assert st["path_samples"] == sum(r["samples"] for r in refs)
    assert st["device_error"] == 0


def test_batch_of_one_cornell_matches_oracle(backend, oracle):
    torch = _torch()
    sb, cam, cfg = cornell_box(0)
    sc = oracle.with_reference_bvh(sb.pack())
    o = oracle.Oracle()
    o_rgb, o_hdr, _ = o.render(sc, cam, cfg, 12345)
    o_dbg = o.debug_read(4, cfg.width * cfg.height)
    h = backend.scene_create(sc)
    try:
        npix = cfg.width * cfg.height
        hdr = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
        rgb = torch.empty(npix * 3, dtype=torch.uint8, device="cuda")
        aux = torch.empty(npix * 2, dtype=torch.int32, device="cuda")
        backend.render_batch([BatchItem(h, cam, cfg, 12345, rgb.data_ptr(), hdr.data_ptr(), aux.data_ptr())])
        assert np.array_equal(aux.cpu().numpy().view(np.uint32), o_dbg)
        assert np.array_equal(hdr.cpu().numpy().view(np.uint32), o_hdr.view(np.uint32))
        assert np.array_equal(rgb.cpu().numpy(), o_rgb)
    finally:
        backend.scene_destroy(h)


def test_batch_rejects_restir_items_and_accepts_empty(backend):
    sb, cam, cfg = sized_field(seed=13, n_tris=2000, width=32, height=32, spp=4, depth=4)
    h = backend.scene_create(sb.pack())
    try:
        backend.render_batch([])
        restir = _cfg(cfg, flags=_abi.RM_FLAG_NO_ENV, restir_spatial=2, restir_candidates=4)
        with pytest.raises(RenderError, match="ReSTIR"):
            backend.render_batch([BatchItem(h, cam, restir, 1)])
        with pytest.raises(RenderError, match="Invalid Metal render dimensions"):
            backend.render_batch([BatchItem(h, cam, _cfg(cfg, spp=0), 1)])
        with pytest.raises(RenderError):
            backend.set_batch_tuning(graph_waves=3)
    finally:
        backend.scene_destroy(h)


def test_tuner_choice_keeps_results(backend, batch_case):
    images, handles, refs = batch_case
    _, _, (items, keep_alive) = _render_batch(backend, images, handles)
    chosen = backend.batch_tune(items)
    del keep_alive
    assert chosen == backend.batch_tuning()
    assert chosen["pool_chunks"] in (32768, 65536, 131072) and chosen["tile_shape"] in (0, 1)
    outs, _, _ = _render_batch(backend, images, handles)
    backend.set_batch_tuning(**TUNINGS[0])
    for o, r in zip(outs, refs):
        assert np.array_equal(o["hdr"].view(np.uint32), r["hdr"].view(np.uint32))
        assert np.array_equal(o["aux"].view(np.uint32), r["aux"])
