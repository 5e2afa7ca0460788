"""ctypes bindings of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` as the checker; the product package never imports it.

* ``liboracle.so`` (oracle/Makefile): the restatement of the reference's
  path (oracle_core.hpp, oracle.cpp).
* ``libref.so`` (oracle/Makefile.ref, optional): the reference's own
  src/engine/{scene,bvh,camera}.cpp compiled where they lie, used to pin the
  restatement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from raymotion_b200 import _abi
from raymotion_b200.scene import Camera, PackedScene, RenderConfig

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libref.so"

_P = C.c_void_p


def build_oracle() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return ORACLE_SO


def reference_root() -> Path | None:
    """The reference checkout that oracle/Makefile.ref reads (the environment
    variable RAYMOTION_REFERENCE overrides the recipe's default), or None when
    it is absent, as on a machine without the checkout."""
    r = subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), "print-ref"], capture_output=True, text=True)
    root = r.stdout.strip() if r.returncode == 0 else ""
    return Path(root) if root and Path(root, "src/engine/bvh.cpp").exists() else None


def build_ref(ref_root: str | None = None) -> Path | None:
    """Compile libref.so from the reference checkout when it is present."""
    root = Path(ref_root) if ref_root else reference_root()
    if root is None or not Path(root, "src/engine/bvh.cpp").exists():
        return REF_SO if REF_SO.exists() else None
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), f"REF={root}"], check=True)
    return REF_SO


def build_dropin(ref_root: str | None = None) -> bool:
    """Build the reference's own test_metal / test_alpha against librmcuda.so
    (the drop-in check) when the reference checkout is present."""
    root = Path(ref_root) if ref_root else reference_root()
    if root is None or not Path(root, "tests/test_metal.cpp").exists():
        return False
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), f"REF={root}", "dropin"], check=True)
    return True


_orc = None
_ref = None


def oracle_lib() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build_oracle()
        lib = C.CDLL(str(ORACLE_SO))
        lib.orc_create.restype = _P
        lib.orc_destroy.argtypes = [_P]
        lib.orc_reset_history.argtypes = [_P]
        lib.orc_render.restype = C.c_int
        lib.orc_render.argtypes = [_P, C.POINTER(_abi.RmSceneView), C.POINTER(_abi.RmCamera),
                                   C.POINTER(_abi.RmConfig), C.c_uint64, _P, _P, C.c_int, C.c_int, C.c_int, _P,
                                   C.c_char_p, C.c_size_t]
        lib.orc_debug_read.restype = C.c_int
        lib.orc_debug_read.argtypes = [_P, C.c_int, _P, C.c_size_t]
        lib.orc_trace.restype = C.c_int
        lib.orc_trace.argtypes = [C.POINTER(_abi.RmSceneView), _P, C.c_int, C.c_int, _P, _P, _P, _P, C.c_int]
        lib.orc_render_f64.restype = C.c_int
        lib.orc_render_f64.argtypes = [C.POINTER(_abi.RmSceneView), C.POINTER(_abi.RmCamera),
                                       C.POINTER(_abi.RmConfig), C.c_uint64, _P, C.c_int, _P, C.c_int]
        lib.orc_render_frozen.restype = C.c_int
        lib.orc_render_frozen.argtypes = [C.POINTER(_abi.RmSceneView), C.POINTER(_abi.RmCamera),
                                          C.POINTER(_abi.RmConfig), C.c_uint64, _P, _P, C.c_int, _P, C.c_int]
        lib.orc_render_frozen_restir.restype = C.c_int
        lib.orc_render_frozen_restir.argtypes = [C.POINTER(_abi.RmSceneView), C.POINTER(_abi.RmCamera),
                                                 C.POINTER(_abi.RmConfig), C.c_uint64, _P, _P, C.c_int, _P,
                                                 C.c_int, C.POINTER(_abi.RmCamera), C.c_uint64]
        lib.orc_build_bvh.restype = C.c_int
        lib.orc_build_bvh.argtypes = [_P, C.c_int, C.c_int, _P, _P, _P]
        lib.orc_refit_bvh.argtypes = [_P, C.c_int, _P, _P, _P]
        lib.orc_detmath.argtypes = [C.c_int, _P, _P, _P, C.c_int]
        _orc = lib
    return _orc


def ref_lib() -> C.CDLL | None:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        lib = C.CDLL(str(REF_SO))
        lib.ref_scene_new.restype = _P
        lib.ref_scene_free.argtypes = [_P]
        lib.ref_add_triangle.restype = C.c_int
        lib.ref_add_triangle.argtypes = [_P, _P, C.c_int]
        lib.ref_tri_count.argtypes = [_P]
        lib.ref_tri_read.argtypes = [_P, _P]
        lib.ref_light_count.argtypes = [_P]
        lib.ref_lights.restype = C.c_double
        lib.ref_lights.argtypes = [_P, _P, _P]
        lib.ref_build_bvh.argtypes = [_P, C.c_int]
        lib.ref_refit_bvh.argtypes = [_P]
        lib.ref_node_count.argtypes = [_P]
        lib.ref_nodes.argtypes = [_P, _P, _P, _P]
        lib.ref_move_vertices.argtypes = [_P, _P]
        lib.ref_append_instance.argtypes = [_P, _P, _P, C.c_int, _P]
        lib.ref_camera.argtypes = [C.c_double] * 7 + [_P]
        _ref = lib
    return _ref


def nthreads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


# ---------------------------------------------------------------- BVH

def build_bvh(verts64: np.ndarray, max_leaf: int = 8):
    """Reference SAH BVH (bvh.cpp restated, fp64): returns (bounds (M,6) f64, links (M,4) i32, bvh_tri)."""
    lib = oracle_lib()
    n = len(verts64)
    if n == 0:
        return np.zeros((0, 6)), np.zeros((0, 4), np.int32), np.zeros(0, np.int32)
    v = np.ascontiguousarray(verts64, np.float64)
    bounds = np.zeros((2 * n, 6))
    links = np.zeros((2 * n, 4), np.int32)
    order = np.zeros(n, np.int32)
    m = lib.orc_build_bvh(v.ctypes.data, n, max_leaf, bounds.ctypes.data, links.ctypes.data, order.ctypes.data)
    return bounds[:m].copy(), links[:m].copy(), order


def refit_bvh(verts64: np.ndarray, bounds: np.ndarray, links: np.ndarray, order: np.ndarray) -> np.ndarray:
    v = np.asarray(verts64, np.float64).reshape(-1, 3, 3)
    tb = np.ascontiguousarray(np.concatenate([v.min(axis=1), v.max(axis=1)], axis=1))
    out = np.ascontiguousarray(bounds.copy())
    oracle_lib().orc_refit_bvh(tb.ctypes.data, len(out), out.ctypes.data, np.ascontiguousarray(links).ctypes.data,
                               np.ascontiguousarray(order).ctypes.data)
    return out


def to_nodes(bounds: np.ndarray, links: np.ndarray) -> np.ndarray:
    """fp64 nodes -> rm_bvh_node records (fp32 boxes), as the Metal host packs them."""
    nodes = np.zeros(len(bounds), _abi.BVH_NODE_DTYPE)
    nodes["mn"] = bounds[:, :3].astype(np.float32)
    nodes["mx"] = bounds[:, 3:].astype(np.float32)
    nodes["left"], nodes["right"], nodes["offset"], nodes["count"] = links.T
    return nodes


def with_reference_bvh(scene: PackedScene, max_leaf: int = 8) -> PackedScene:
    """Attach the reference-rule SAH BVH (as Scene::nodes would hold it)."""
    b, l, o = build_bvh(scene.verts64, max_leaf)
    scene.nodes = to_nodes(b, l)
    scene.bvh_tri = o
    return scene


# ---------------------------------------------------------------- render

class Oracle:
    def __init__(self):
        self.lib = oracle_lib()
        self.h = self.lib.orc_create()

    def __del__(self):
        try:
            self.lib.orc_destroy(self.h)
        except Exception:
            pass

    def reset_history(self):
        self.lib.orc_reset_history(self.h)

    def render(self, scene: PackedScene, cam: Camera, cfg: RenderConfig, seed: int = 12345, threads: int | None = None,
               rows: tuple[int, int] | None = None):
        """Returns (rgb u8[W*H*3], hdr f32[W*H*3], stats dict).  The scene must carry a BVH."""
        assert scene.nodes is not None or scene.n_tris == 0, "the oracle traverses a caller BVH"
        npix = cfg.width * cfg.height
        rgb = np.zeros(npix * 3, np.uint8)
        hdr = np.zeros(npix * 3, np.float32)
        st = np.zeros(3, np.uint64)
        v = scene.view(True)
        e = C.create_string_buffer(512)
        r0, r1 = rows if rows else (0, 0)
        rc = self.lib.orc_render(self.h, C.byref(v), C.byref(cam.packed()), C.byref(cfg.packed()),
                                 C.c_uint64(seed & 0xFFFFFFFFFFFFFFFF), rgb.ctypes.data, hdr.ctypes.data,
                                 threads or nthreads(), r0, r1, st.ctypes.data, e, 512)
        if rc != 0:
            raise RuntimeError(e.value.decode())
        return rgb, hdr, dict(path_samples=int(st[0]), rays=int(st[1]), chain=int(st[2]))

    def debug_read(self, which: int, npix: int) -> np.ndarray:
        dt = {0: _abi.GBUF_DTYPE, 1: _abi.RESERVOIR_DTYPE, 2: _abi.RESERVOIR_DTYPE, 3: np.float32, 4: np.uint32}[which]
        count = npix * (3 if which == 3 else 2 if which == 4 else 1)
        out = np.zeros(count, dt)
        rc = self.lib.orc_debug_read(self.h, which, out.ctypes.data, out.nbytes)
        if rc != 0:
            raise RuntimeError("oracle debug read failed")
        return out


def trace(scene: PackedScene, rays: np.ndarray, any_hit: bool = False, threads: int | None = None):
    n = len(rays)
    r = np.ascontiguousarray(rays, np.float32)
    tri = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    sv = scene.view(True)
    oracle_lib().orc_trace(C.byref(sv), r.ctypes.data, n, int(any_hit), tri.ctypes.data, t.ctypes.data,
                           u.ctypes.data, v.ctypes.data, threads or nthreads())
    return tri, t, u, v


def render_f64(scene: PackedScene, cam: Camera, cfg: RenderConfig, seed: int, pixels: np.ndarray | None = None,
               threads: int | None = None) -> np.ndarray:
    n = len(pixels) if pixels is not None else cfg.width * cfg.height
    out = np.zeros((n, 3), np.float64)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.int32)
    sv = scene.view(True)
    oracle_lib().orc_render_f64(C.byref(sv), C.byref(cam.packed()), C.byref(cfg.packed()),
                                C.c_uint64(seed), out.ctypes.data, threads or nthreads(),
                                None if px is None else px.ctypes.data, n)
    return out


def render_frozen(scene: PackedScene, cam: Camera, cfg: RenderConfig, seed: int, tri_material: np.ndarray,
                  params: np.ndarray, threads: int | None = None) -> np.ndarray:
    """The plain frame with its paths frozen at the scene's own materials and the
    material factors evaluated in double at ``params`` (n_materials x 8:
    albedo rgb, rough, emission rgb, ior) through ``tri_material``; W*H x 3."""
    tm = np.ascontiguousarray(tri_material, np.int32)
    prm = np.ascontiguousarray(params, np.float64)
    assert len(tm) == scene.n_tris and prm.ndim == 2 and prm.shape[1] == 8
    out = np.zeros((cfg.width * cfg.height, 3), np.float64)
    sv = scene.view(True)
    rc = oracle_lib().orc_render_frozen(C.byref(sv), C.byref(cam.packed()), C.byref(cfg.packed()), C.c_uint64(seed),
                                        tm.ctypes.data, prm.ctypes.data, len(prm), out.ctypes.data,
                                        threads or nthreads())
    if rc != 0:
        raise ValueError("frozen evaluation needs a fixed sample count and the plain chain")
    return out


def render_frozen_restir(scene: PackedScene, cam: Camera, cfg: RenderConfig, seed: int, tri_material: np.ndarray,
                         params: np.ndarray, threads: int | None = None, prev: tuple[Camera, int] | None = None
                         ) -> np.ndarray:
    """The ReSTIR frame with K3/K4 run at the scene's own materials and held,
    K5 replayed frozen with the material factors in double at ``params``, and
    the denoiser (unless the config turns it off) in double on the held
    G-buffers; W*H x 3.  ``prev`` = (camera, seed) of the frame before it (its
    history, rendered in fp32), else the first frame of a history."""
    tm = np.ascontiguousarray(tri_material, np.int32)
    prm = np.ascontiguousarray(params, np.float64)
    assert len(tm) == scene.n_tris and prm.ndim == 2 and prm.shape[1] == 8
    out = np.zeros((cfg.width * cfg.height, 3), np.float64)
    sv = scene.view(True)
    pcam = C.byref(prev[0].packed()) if prev else None
    rc = oracle_lib().orc_render_frozen_restir(C.byref(sv), C.byref(cam.packed()), C.byref(cfg.packed()),
                                               C.c_uint64(seed), tm.ctypes.data, prm.ctypes.data, len(prm),
                                               out.ctypes.data, threads or nthreads(), pcam,
                                               C.c_uint64(prev[1] if prev else 0))
    if rc != 0:
        raise ValueError("frozen ReSTIR evaluation needs a configuration the policy renders with ReSTIR")
    return out


def detmath(which: int, x: np.ndarray):
    x = np.ascontiguousarray(x, np.float32)
    y0 = np.zeros_like(x)
    y1 = np.zeros_like(x)
    oracle_lib().orc_detmath(which, x.ctypes.data, y0.ctypes.data, y1.ctypes.data, len(x))
    return y0, y1
