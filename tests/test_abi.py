"""librmcuda.so loads without a GPU and exports every function include/rmcuda.h declares."""
import ctypes as C
import re
from pathlib import Path

import pytest

import raymotion_b200 as rb
from raymotion_b200 import _abi, build

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "rmcuda.h").read_text()
    return sorted(set(re.findall(r"\b(rmcuda_[a-z_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not build.LIB.exists():
        build.build()
    return _abi.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 14
    bound = {n for n, _, _ in _abi.EXPORTS}
    for n in names:
        assert hasattr(lib, n), n
        assert n in bound, f"{n} lacks a ctypes binding"


def test_checked_build_exports_the_same_symbols():
    """librmcuda_checked.so (device-side bounds checks, RMCUDA_CHECKED) loads
    and exports every declared symbol, and RAYMOTION_CUDA_CHECKED=1 selects it."""
    import os
    import subprocess
    import sys
    from raymotion_b200 import build
    if not build.LIB_CHECKED.exists():
        build.build(checked=True)
    lib = _abi.load_library(build.LIB_CHECKED)
    for n in _declared():
        assert hasattr(lib, n), n
    code = ("import raymotion_b200._abi as a; a.load_library(); "
            "print([l for l in open('/proc/self/maps') if 'librmcuda' in l][0].split()[-1])")
    env = dict(os.environ, RAYMOTION_CUDA_CHECKED="1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, cwd=str(build.ROOT),
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip().splitlines()[-1].endswith("librmcuda_checked.so")


def test_record_sizes_match_reference_abi():
    # metal_types.h sizes, asserted in metal.mm:13-17
    assert _abi.TRIANGLE_DTYPE.itemsize == 176
    assert _abi.GBUF_DTYPE.itemsize == 76
    assert _abi.RESERVOIR_DTYPE.itemsize == 60
    assert C.sizeof(_abi.RmCamera) == 52


def test_version_and_unavailable_without_gpu(lib):
    assert lib.rmcuda_version().startswith(b"rmcuda")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    rc = lib.rmcuda_create(C.byref(h), 0, err, 256)
    assert rc == _abi.RM_ERR_UNAVAILABLE
    # the reference test suite treats this exact string as "skip" (tests/test_metal.cpp:25)
    assert err.value == b"Metal backend is not available in this build"


def test_render_image_metal_validates_first():
    from raymotion_b200.scene import Camera, RenderConfig, SceneBuilder
    ok, rgb, err = rb.render_image_metal(SceneBuilder().pack(), Camera(), RenderConfig(width=0), 1)
    assert not ok and err == "Invalid Metal render dimensions or sample count"


def test_preview_channel_framing():
    """rmcuda_preview_frame (no GPU): the frame line and bytes of the
    reference's preview channel, then one granted byte per frame; end of file
    on the grant descriptor ends the preview, a closed channel is an error."""
    import os

    import numpy as np

    import raymotion_b200 as rb
    rgb = (np.arange(4 * 3 * 3) % 256).astype(np.uint8)
    r, w = os.pipe()
    gr, gw = os.pipe()
    os.write(gw, b"x")
    assert rb.preview_frame(w, rgb, 4, 3, 7, gr)
    os.close(w)
    data = os.read(r, 1 << 16)
    head, body = data.split(b"\n", 1)
    assert head == b"RAY1 4 3 7 36" and body == rgb.tobytes()
    os.close(gw)  # no further grant: the preview is complete
    r2, w2 = os.pipe()
    assert not rb.preview_frame(w2, rgb, 4, 3, 8, gr)
    os.close(r2)
    os.close(gr)
    with pytest.raises(rb.RenderError, match="preview channel closed"):
        rb.preview_frame(w2, rgb, 4, 3, 9)
    os.close(w2)
    os.close(r)
