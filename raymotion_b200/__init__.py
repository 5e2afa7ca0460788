"""raymotion_b200 - B200 (sm_100a) backend for raymotion's path-tracing hot path.

The native library ``librmcuda.so`` (CUDA kernels + the C ABI of
include/rmcuda.h) does the work; this module is a thin host-side mirror of the
reference's backend entry point

    bool render_image_metal(const Scene&, const Camera&, const RenderConfig&,
                            uint64_t seed, std::vector<uint8_t>& rgb, std::string& error)

(reference include/raymotion/metal.hpp:6-7): ``render_image_metal`` returns
``(ok, rgb, error)`` with the same error strings, and ``Backend`` exposes the
context, the device-resident scene and the traversal queries used by the
benchmark and the parity tests.  There is no CPU fallback: without the
library or a sm_100 GPU every call fails loudly.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import GBUF_DTYPE, RESERVOIR_DTYPE, load_library
from .scene import Camera, PackedScene, RenderConfig, SceneBuilder, Texture

__all__ = ["Backend", "BatchItem", "RenderError", "render_image_metal", "Camera", "RenderConfig", "SceneBuilder",
           "Texture", "PackedScene", "load_library"]


class RenderError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def _err() -> C.Array:
    return C.create_string_buffer(512)


@dataclass
class BatchItem:
    """One image of a batch (rm_batch_item): a scene object, its view and config,
    and DEVICE output pointers (RGB8 W*H*3, radiance W*H*3 floats, and per
    pixel (xor of the final lane RNG states, samples taken)), any may be None."""
    scene: int
    camera: Camera
    config: RenderConfig
    seed: int = 12345
    d_rgb: int | None = None
    d_hdr: int | None = None
    d_aux: int | None = None


def _batch_array(items) -> C.Array:
    arr = (_abi.RmBatchItem * max(len(items), 1))()
    for k, it in enumerate(items):
        a = arr[k]
        a.scene = it.scene
        a.camera = it.camera.packed()
        a.config = it.config.packed()
        a.seed = it.seed & 0xFFFFFFFFFFFFFFFF
        a.d_rgb = it.d_rgb
        a.d_hdr = it.d_hdr
        a.d_aux = it.d_aux
    return arr


class Backend:
    """One rmcuda context on a CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        e = _err()
        rc = self.lib.rmcuda_create(C.byref(h), device, e, 512)
        if rc != _abi.RM_OK:
            raise RenderError(rc, e.value.decode())
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.rmcuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, e) -> None:
        if rc != _abi.RM_OK:
            raise RenderError(rc, e.value.decode())

    # ---- whole frame through the reference-facing call (host buffers)
    def render(self, scene: PackedScene, cam: Camera, cfg: RenderConfig, seed: int = 12345, hdr: bool = False,
               use_nodes: bool = True, out: np.ndarray | None = None):
        """One synchronous frame; ``out`` (uint8, W*H*3) receives the image when given."""
        npix = cfg.width * cfg.height
        rgb = out if out is not None else np.empty(max(npix, 0) * 3, np.uint8)
        out_hdr = np.empty(max(npix, 0) * 3, np.float32) if hdr else None
        v = scene.view(use_nodes)
        e = _err()
        rc = self.lib.rmcuda_render(self.h, C.byref(v), C.byref(cam.packed()), C.byref(cfg.packed()),
                                    C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), _abi.ptr(rgb), rgb.nbytes,
                                    _abi.ptr(out_hdr), e, 512)
        self._check(rc, e)
        return (rgb, out_hdr) if hdr else rgb

    # ---- device-resident scene
    def upload(self, scene: PackedScene, use_nodes: bool = True) -> None:
        v = scene.view(use_nodes)
        e = _err()
        self._check(self.lib.rmcuda_scene_upload(self.h, C.byref(v), e, 512), e)

    def update(self, tris: np.ndarray, rebuild_every: int = 0) -> None:
        e = _err()
        self._check(self.lib.rmcuda_scene_update(self.h, _abi.ptr(tris), len(tris), rebuild_every, e, 512), e)

    # ---- device-side scene preparation (Objects on the device)
    def model_create(self, tris: np.ndarray) -> int:
        """Upload object-space model triangles (MODEL_TRI_DTYPE); returns the model id."""
        tris = np.ascontiguousarray(tris, _abi.MODEL_TRI_DTYPE)
        mid = C.c_int32(-1)
        e = _err()
        self._check(self.lib.rmcuda_model_create(self.h, _abi.ptr(tris), len(tris), C.byref(mid), e, 512), e)
        return int(mid.value)

    def model_update(self, model: int, tris: np.ndarray) -> None:
        tris = np.ascontiguousarray(tris, _abi.MODEL_TRI_DTYPE)
        e = _err()
        self._check(self.lib.rmcuda_model_update(self.h, int(model), _abi.ptr(tris), len(tris), e, 512), e)

    def instances_commit(self, inst: np.ndarray, rebuild_every: int = 32) -> None:
        """Build the world of ``inst`` (INSTANCE_DTYPE) on the device and make it the resident scene."""
        inst = np.ascontiguousarray(inst, _abi.INSTANCE_DTYPE)
        e = _err()
        self._check(self.lib.rmcuda_instances_commit(self.h, _abi.ptr(inst), len(inst), int(rebuild_every), e, 512),
                    e)

    def scene_read(self):
        """The resident scene: (triangles, light_tri, light_cdf, light_total)."""
        counts = np.zeros(2, np.int32)
        tot = C.c_float(0)
        e = _err()
        self._check(self.lib.rmcuda_scene_read(self.h, None, 0, None, None, 0, _abi.ptr(counts), C.byref(tot), e, 512),
                    e)
        tris = np.zeros(int(counts[0]), _abi.TRIANGLE_DTYPE)
        lt = np.zeros(int(counts[1]), np.int32)
        cdf = np.zeros(int(counts[1]), np.float32)
        self._check(self.lib.rmcuda_scene_read(self.h, _abi.ptr(tris), len(tris), _abi.ptr(lt), _abi.ptr(cdf), len(lt),
                                               _abi.ptr(counts), C.byref(tot), e, 512), e)
        return tris, lt, cdf, np.float32(tot.value)

    def render_resident_async(self, cam: Camera, cfg: RenderConfig, seed: int, d_rgb: int | None,
                              d_hdr: int | None = None) -> None:
        e = _err()
        self._check(self.lib.rmcuda_render_resident_async(self.h, C.byref(cam.packed()), C.byref(cfg.packed()),
                                                          C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), d_rgb, d_hdr, e,
                                                          512), e)

    def sync(self) -> None:
        e = _err()
        self._check(self.lib.rmcuda_sync(self.h, e, 512), e)

    def set_stream(self, stream_handle: int | None) -> None:
        e = _err()
        self._check(self.lib.rmcuda_set_stream(self.h, stream_handle, e, 512), e)

    def trace(self, d_rays: int, n: int, any_hit: bool, d_tri: int, d_t: int | None = None, d_u: int | None = None,
              d_v: int | None = None) -> None:
        e = _err()
        self._check(self.lib.rmcuda_trace(self.h, d_rays, n, int(any_hit), d_tri, d_t, d_u, d_v, e, 512), e)

    def debug_read(self, which: int, npix: int) -> np.ndarray:
        dt = {0: GBUF_DTYPE, 1: RESERVOIR_DTYPE, 2: RESERVOIR_DTYPE, 3: np.float32, 4: np.uint32}[which]
        count = npix * (3 if which == 3 else 2 if which == 4 else 1)
        out = np.empty(count, dt)
        e = _err()
        self._check(self.lib.rmcuda_debug_read(self.h, which, _abi.ptr(out), out.nbytes, e, 512), e)
        return out

    # ---- scene objects and batched rendering
    def scene_create(self, scene: PackedScene, use_nodes: bool = False) -> int:
        """Upload a scene into buffers of its own; returns its handle."""
        v = scene.view(use_nodes)
        h = C.c_void_p()
        e = _err()
        self._check(self.lib.rmcuda_scene_create(self.h, C.byref(v), C.byref(h), e, 512), e)
        return h.value

    def scene_destroy(self, handle: int) -> None:
        self.lib.rmcuda_scene_destroy(self.h, handle)

    def render_scene_async(self, handle: int, cam: Camera, cfg: RenderConfig, seed: int, d_rgb: int | None,
                           d_hdr: int | None = None) -> None:
        """The single-frame policy on a scene object, into device buffers (not waited for)."""
        e = _err()
        self._check(self.lib.rmcuda_render_scene_async(self.h, handle, C.byref(cam.packed()), C.byref(cfg.packed()),
                                                       C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), d_rgb, d_hdr, e, 512),
                    e)

    def render_batch(self, items) -> None:
        """Render a list of BatchItem together (synchronous)."""
        arr = _batch_array(items)
        e = _err()
        self._check(self.lib.rmcuda_render_batch(self.h, arr, len(items), e, 512), e)

    def batch_tune(self, items) -> dict:
        """Pick launch settings on the first waves of this batch; returns them."""
        arr = _batch_array(items)
        t = _abi.RmBatchTuning()
        e = _err()
        self._check(self.lib.rmcuda_batch_tune(self.h, arr, len(items), C.byref(t), e, 512), e)
        return {f: getattr(t, f) for f, _ in _abi.RmBatchTuning._fields_}

    def batch_log(self) -> np.ndarray:
        """(live lane slots, extension rays) at each progress check of the last batch."""
        n = self.lib.rmcuda_batch_log(self.h, None, 0)
        out = np.zeros((max(n, 0), 2), np.int32)
        if n > 0:
            self.lib.rmcuda_batch_log(self.h, out.ctypes.data_as(C.POINTER(C.c_int32)), n)
        return out

    def batch_tuning(self) -> dict:
        t = _abi.RmBatchTuning()
        self.lib.rmcuda_batch_get_tuning(self.h, C.byref(t))
        return {f: getattr(t, f) for f, _ in _abi.RmBatchTuning._fields_}

    def set_batch_tuning(self, **kw) -> None:
        t = _abi.RmBatchTuning(**{**self.batch_tuning(), **kw})
        e = _err()
        self._check(self.lib.rmcuda_batch_set_tuning(self.h, C.byref(t), e, 512), e)

    # ---- differentiable rendering
    def scene_set_materials(self, handle: int, params: np.ndarray, tri_material: np.ndarray | None = None,
                            light_cdf: np.ndarray | None = None, light_total: float = 0.0) -> None:
        """Per-triangle materials of a scene object (params: n x 8 float32)."""
        prm = np.ascontiguousarray(params, np.float32)
        assert prm.ndim == 2 and prm.shape[1] == 8
        tm = None if tri_material is None else np.ascontiguousarray(tri_material, np.int32)
        cdf = None if light_cdf is None else np.ascontiguousarray(light_cdf, np.float32)
        e = _err()
        self._check(self.lib.rmcuda_scene_set_materials(self.h, handle, _abi.ptr(tm), _abi.ptr(prm), len(prm),
                                                         _abi.ptr(cdf), float(light_total), e, 512), e)

    def backward(self, handle: int, cam: Camera, cfg: RenderConfig, seed: int, d_dl_dimage: int,
                 d_grad: int) -> None:
        """Path-replay adjoint: adds dL/dparams (device, n x 8 floats) given dL/dimage (device)."""
        e = _err()
        self._check(self.lib.rmcuda_backward(self.h, handle, C.byref(cam.packed()), C.byref(cfg.packed()),
                                             C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), d_dl_dimage, d_grad, e, 512), e)

    def preview_last(self, fd: int, frame: int, grant_fd: int = -1) -> bool:
        """Write the last frame to the preview channel `fd` (RAY1 framing); with
        grant_fd, wait for one byte there.  False when grant_fd is at end of file."""
        e = _err()
        rc = self.lib.rmcuda_preview_last(self.h, fd, frame, grant_fd, e, 512)
        if rc == _abi.RM_PREVIEW_DONE:
            return False
        self._check(rc, e)
        return True

    def reset_history(self) -> None:
        self.lib.rmcuda_reset_history(self.h)

    def stats(self) -> dict:
        s = _abi.RmStats()
        rc = self.lib.rmcuda_stats_get(self.h, C.byref(s))
        if rc != _abi.RM_OK:
            raise RenderError(rc, "stats read failed")
        return dict(path_samples=s.path_samples, rays=s.rays, nodes_visited=s.nodes_visited,
                    tris_tested=s.tris_tested, frames=s.frames, kernel_launches=s.kernel_launches,
                    device_error=s.device_error, kernel_chain=s.kernel_chain, bvh_node_bytes=s.bvh_node_bytes,
                    bvh_builds=s.bvh_builds, bvh_refits=s.bvh_refits, bvh_kept=s.bvh_kept)

    def stats_reset(self) -> None:
        self.lib.rmcuda_stats_reset(self.h)

    def profile(self, level: int = 1) -> None:
        self.lib.rmcuda_profile(self.h, int(level))

    def stage_times(self) -> dict:
        n = len(_abi.STAGES)
        ms = (C.c_double * n)()
        cnt = (C.c_uint64 * n)()
        self.lib.rmcuda_stage_times(self.h, ms, cnt, n)
        return {name: (ms[i], int(cnt[i])) for i, name in enumerate(_abi.STAGES)}

    def wave_log(self) -> np.ndarray:
        """(act, ext, shd, us) per count read (every 4 waves) of the last wavefront frame."""
        n = self.lib.rmcuda_wave_log(self.h, None, 0)
        out = np.zeros((max(n, 0), 4), np.int32)
        if n > 0:
            self.lib.rmcuda_wave_log(self.h, out.ctypes.data_as(C.POINTER(C.c_int32)), n)
        return out

    def stage_counters(self) -> dict:
        n = len(_abi.STAGES)
        out = (C.c_uint64 * (4 * n))()
        rc = self.lib.rmcuda_stage_counters(self.h, out, n)
        if rc != _abi.RM_OK:
            raise RenderError(rc, "counter read failed")
        return {name: dict(path_samples=int(out[4 * i]), rays=int(out[4 * i + 1]), nodes_visited=int(out[4 * i + 2]),
                           tris_tested=int(out[4 * i + 3])) for i, name in enumerate(_abi.STAGES)}


_default: Backend | None = None
_default_error: RenderError | None = None


def render_image_metal(scene: PackedScene, cam: Camera, cfg: RenderConfig, seed: int = 12345):
    """Python mirror of render_image_metal: returns (ok, rgb, error)."""
    global _default, _default_error
    if cfg.width <= 0 or cfg.height <= 0 or cfg.spp <= 0 or cfg.max_bounces < 0 or cfg.width * cfg.height > 100000000:
        return False, np.zeros(0, np.uint8), "Invalid Metal render dimensions or sample count"
    if _default is None and _default_error is None:
        try:
            _default = Backend(0)
        except (RenderError, OSError) as ex:
            _default_error = ex if isinstance(ex, RenderError) else RenderError(_abi.RM_ERR_UNAVAILABLE, str(ex))
    if _default is None:
        return False, np.zeros(0, np.uint8), str(_default_error)
    try:
        return True, _default.render(scene, cam, cfg, seed), ""
    except RenderError as ex:
        return False, np.zeros(0, np.uint8), str(ex)


def preview_frame(fd: int, rgb: np.ndarray, width: int, height: int, frame: int, grant_fd: int = -1) -> bool:
    """Write a host RGB8 image to the preview channel `fd` ("RAY1 w h frame
    bytes" line, then the bytes; include/raymotion/preview.hpp:17-23).  With
    grant_fd, wait for one byte there; False when it is at end of file."""
    buf = np.ascontiguousarray(rgb, np.uint8)
    assert buf.size == width * height * 3
    lib = _abi.load_library()
    e = _err()
    rc = lib.rmcuda_preview_frame(fd, _abi.ptr(buf), width, height, frame, grant_fd, e, 512)
    if rc == _abi.RM_PREVIEW_DONE:
        return False
    if rc != _abi.RM_OK:
        raise RenderError(rc, e.value.decode())
    return True
