"""ctypes view of the C ABI declared in include/rmcuda.h.

The record layouts are the reference's Metal ABI (src/engine/metal_types.h):
a packed 176-byte triangle, a 52-byte camera, and the reference ReSTIR
G-buffer (76 B) and reservoir (60 B) records used by the debug reads.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "librmcuda.so"

RM_OK = 0
RM_ERR_INVALID = 1
RM_ERR_UNAVAILABLE = 2
RM_ERR_CUDA = 3
RM_ERR_ALLOC = 4
RM_ERR_BVH = 5
RM_ERR_DEVICE = 6
RM_PREVIEW_DONE = 7  # the preview grant descriptor reached end of file

RM_FLAG_NO_ENV = 0x1
RM_FLAG_NOADAPT = 0x2
RM_FLAG_NOMIS = 0x4
RM_FLAG_RESTIR_OFF = 0x8
RM_FLAG_DENOISE_OFF = 0x10
RM_FLAG_TEMPORAL_OFF = 0x20
RM_FLAG_NO_RR = 0x40
RM_FLAG_ANIMATED_HISTORY = 0x100

_v3 = [("x", "<f4"), ("y", "<f4"), ("z", "<f4")]
TRIANGLE_DTYPE = np.dtype(
    [(name, "<f4", (3,)) for name in ("v0", "v1", "v2", "n", "nn", "n0", "n1", "n2")]
    + [(name, "<f4") for name in ("ar", "ag", "ab", "er", "eg", "eb", "ior", "rough", "metallic", "alpha")]
    + [("shader", "<i4")]
    + [(name, "<f4") for name in ("tu0", "tv0", "tu1", "tv1", "tu2", "tv2")]
    + [("texture_offset", "<i4"), ("texture_width", "<i4"), ("texture_height", "<i4")]
)
assert TRIANGLE_DTYPE.itemsize == 176

# rm_model_tri / rm_instance (include/rmcuda.h): object-space model triangles
# and instances of the device-side scene preparation
MODEL_TRI_DTYPE = np.dtype([(k, "<f8", (3,)) for k in ("v0", "v1", "v2", "n0", "n1", "n2")]
                           + [(k, "<f8") for k in ("tu0", "tv0", "tu1", "tv1", "tu2", "tv2", "ar", "ag", "ab", "er",
                                                   "eg", "eb", "metallic", "ior", "rough", "alpha")]
                           + [("shader", "<i4"), ("reserved", "<i4")])
assert MODEL_TRI_DTYPE.itemsize == 280
INSTANCE_DTYPE = np.dtype([("model", "<i4"), ("reserved", "<i4")]
                          + [(k, "<f8", (3,)) for k in ("position", "cos_rot", "sin_rot", "scale", "albedo",
                                                        "emission")]
                          + [(k, "<f8") for k in ("refract", "rough", "metallic", "alpha")])
assert INSTANCE_DTYPE.itemsize == 184

BVH_NODE_DTYPE = np.dtype([("mn", "<f4", (3,)), ("mx", "<f4", (3,)), ("left", "<i4"), ("right", "<i4"),
                           ("offset", "<i4"), ("count", "<i4")])
assert BVH_NODE_DTYPE.itemsize == 40

GBUF_DTYPE = np.dtype([("pos", "<f4", (3,)), ("normal", "<f4", (3,)), ("albedo", "<f4", (3,)),
                       ("wo", "<f4", (3,)), ("emission", "<f4", (3,)), ("rough", "<f4"), ("metallic", "<f4"),
                       ("ior", "<f4"), ("kind", "<i4")])
assert GBUF_DTYPE.itemsize == 76
RESERVOIR_DTYPE = np.dtype([("lightPos", "<f4", (3,)), ("lightNormal", "<f4", (3,)), ("emission", "<f4", (3,)),
                            ("alpha", "<f4"), ("p_hat", "<f4"), ("sumWs", "<f4"), ("sumWu", "<f4"),
                            ("M", "<u4"), ("valid", "<u4")])
assert RESERVOIR_DTYPE.itemsize == 60


class RmCamera(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("x", "y", "z", "focal", "m0", "m1", "m2", "m3", "m4", "m5", "m6", "m7", "m8")]


class RmSceneView(C.Structure):
    _fields_ = [
        ("tris", C.c_void_p), ("n_tris", C.c_int32), ("n_nodes", C.c_int32), ("nodes", C.c_void_p),
        ("bvh_tri", C.c_void_p), ("light_tri", C.c_void_p), ("light_cdf", C.c_void_p), ("n_lights", C.c_int32),
        ("light_total", C.c_float), ("texels", C.c_void_p), ("n_texels", C.c_int64),
    ]


class RmConfig(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_bounces", C.c_int32),
        ("resolution", C.c_float), ("clamp", C.c_float), ("adapt_rel", C.c_float), ("adapt_abs", C.c_float),
        ("adapt_min", C.c_int32), ("adapt_step", C.c_int32), ("restir_candidates", C.c_int32),
        ("restir_spatial", C.c_int32), ("restir_radius", C.c_float), ("restir_mcap", C.c_int32),
        ("flags", C.c_uint32),
    ]


class RmStats(C.Structure):
    _fields_ = [("path_samples", C.c_uint64), ("rays", C.c_uint64), ("nodes_visited", C.c_uint64),
                ("tris_tested", C.c_uint64), ("frames", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("device_error", C.c_uint32), ("kernel_chain", C.c_uint32), ("bvh_node_bytes", C.c_uint32),
                ("bvh_builds", C.c_uint32), ("bvh_refits", C.c_uint32), ("bvh_kept", C.c_uint32)]


class RmBatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", RmCamera), ("config", RmConfig), ("seed", C.c_uint64),
                ("d_rgb", C.c_void_p), ("d_hdr", C.c_void_p), ("d_aux", C.c_void_p)]


class RmBatchTuning(C.Structure):
    _fields_ = [("pool_chunks", C.c_int32), ("tile_shape", C.c_int32), ("grid_scale", C.c_int32),
                ("graph_waves", C.c_int32), ("bvh_width", C.c_int32)]


# (name, restype, argtypes) of every symbol declared in include/rmcuda.h
_P = C.c_void_p
_S = C.c_char_p
_Z = C.c_size_t
EXPORTS = [
    ("rmcuda_version", C.c_char_p, []),
    ("rmcuda_create", C.c_int, [C.POINTER(_P), C.c_int, _S, _Z]),
    ("rmcuda_destroy", None, [_P]),
    ("rmcuda_set_stream", C.c_int, [_P, _P, _S, _Z]),
    ("rmcuda_render", C.c_int, [_P, C.POINTER(RmSceneView), C.POINTER(RmCamera), C.POINTER(RmConfig), C.c_uint64,
                                _P, _Z, _P, _S, _Z]),
    ("rmcuda_scene_upload", C.c_int, [_P, C.POINTER(RmSceneView), _S, _Z]),
    ("rmcuda_scene_update", C.c_int, [_P, _P, C.c_int32, C.c_int32, _S, _Z]),
    ("rmcuda_model_create", C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32), _S, _Z]),
    ("rmcuda_model_update", C.c_int, [_P, C.c_int32, _P, C.c_int32, _S, _Z]),
    ("rmcuda_instances_commit", C.c_int, [_P, _P, C.c_int32, C.c_int32, _S, _Z]),
    ("rmcuda_scene_read", C.c_int, [_P, _P, C.c_int32, _P, _P, C.c_int32, _P, C.POINTER(C.c_float), _S, _Z]),
    ("rmcuda_preview_frame", C.c_int, [C.c_int32, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _S, _Z]),
    ("rmcuda_preview_last", C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _S, _Z]),
    ("rmcuda_render_resident_async", C.c_int, [_P, C.POINTER(RmCamera), C.POINTER(RmConfig), C.c_uint64, _P, _P,
                                                _S, _Z]),
    ("rmcuda_sync", C.c_int, [_P, _S, _Z]),
    ("rmcuda_trace", C.c_int, [_P, _P, C.c_int32, C.c_int32, _P, _P, _P, _P, _S, _Z]),
    ("rmcuda_debug_read", C.c_int, [_P, C.c_int32, _P, _Z, _S, _Z]),
    ("rmcuda_reset_history", C.c_int, [_P]),
    ("rmcuda_stats_get", C.c_int, [_P, C.POINTER(RmStats)]),
    ("rmcuda_stats_reset", C.c_int, [_P]),
    ("rmcuda_profile", C.c_int, [_P, C.c_int]),
    ("rmcuda_stage_counters", C.c_int, [_P, C.POINTER(C.c_uint64), C.c_int32]),
    ("rmcuda_wave_log", C.c_int, [_P, C.POINTER(C.c_int32), C.c_int32]),
    ("rmcuda_trace_noalloc", C.c_int, [_P, C.c_int32, _P, C.c_int32, C.c_int32, _P, _P, _P, _P, _P, _S, _Z]),
    ("rmcuda_stage_times", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.c_int32]),
    ("rmcuda_scene_create", C.c_int, [_P, C.POINTER(RmSceneView), C.POINTER(_P), _S, _Z]),
    ("rmcuda_scene_destroy", None, [_P, _P]),
    ("rmcuda_render_scene_async", C.c_int, [_P, _P, C.POINTER(RmCamera), C.POINTER(RmConfig), C.c_uint64, _P, _P,
                                             _S, _Z]),
    ("rmcuda_render_batch", C.c_int, [_P, C.POINTER(RmBatchItem), C.c_int32, _S, _Z]),
    ("rmcuda_batch_tune", C.c_int, [_P, C.POINTER(RmBatchItem), C.c_int32, C.POINTER(RmBatchTuning), _S, _Z]),
    ("rmcuda_batch_log", C.c_int, [_P, C.POINTER(C.c_int32), C.c_int32]),
    ("rmcuda_scene_set_materials", C.c_int, [_P, _P, _P, _P, C.c_int32, _P, C.c_float, _S, _Z]),
    ("rmcuda_backward", C.c_int, [_P, _P, C.POINTER(RmCamera), C.POINTER(RmConfig), C.c_uint64, _P, _P, _S, _Z]),
    ("rmcuda_batch_get_tuning", C.c_int, [_P, C.POINTER(RmBatchTuning)]),
    ("rmcuda_batch_set_tuning", C.c_int, [_P, C.POINTER(RmBatchTuning), _S, _Z]),
]

STAGES = ["plain", "hash", "generate", "spatial", "shade", "temporal", "atrous0", "atrous1", "tonemap", "wf_extend",
          "wf_shadow", "wf_shade", "bt_start", "bt_extend", "bt_shadow", "bt_shade", "batch", "adjoint",
          "wf_tail", "prep"]

_lib = None


def load_library(path: Path | str | None = None) -> C.CDLL:
    """Load librmcuda.so (built in-tree by raymotion_b200.build) and bind its symbols.

    Raises OSError if the library is missing: there is no fallback path.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    default = LIB_PATH
    if os.environ.get("RAYMOTION_CUDA_CHECKED") == "1":
        default = LIB_PATH.with_name("librmcuda_checked.so")  # device-side bounds checks (build.py checked)
    p = Path(path) if path else default
    if not p.exists():
        raise OSError(f"{p} is missing; run raymotion_b200.build.build() first")
    lib = C.CDLL(str(p))
    for name, res, args in EXPORTS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays crossing the ABI must be C-contiguous"
    return a.ctypes.data
