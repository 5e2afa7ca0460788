"""The reference's own backend tests, linked against librmcuda.so in place of
the Metal backend (oracle/Makefile.ref `dropin`: tests/test_metal.cpp and
tests/test_alpha.cpp plus the reference engine, compiled from the reference
tree against its own headers)."""
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "oracle" / "_ref"


def _bin(name):
    p = BIN / name
    if not p.exists():
        pytest.skip(f"{p} not built (oracle/Makefile.ref dropin needs the reference checkout)")
    return p


def _cuda_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_test_metal_skips_without_gpu():
    if _cuda_visible():
        pytest.skip("a GPU is present")
    r = subprocess.run([str(_bin("test_metal_dropin"))], capture_output=True, text=True, timeout=60)
    assert r.returncode == 77, r.stderr  # SKIP_RETURN_CODE of the reference's ctest registration
    assert "Metal backend is not available in this build" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["test_metal_dropin", "test_alpha_dropin"])
def test_reference_backend_tests_pass_on_gpu(name):
    env = dict(os.environ, RAYMOTION_REQUIRE_METAL="1")
    r = subprocess.run([str(_bin(name))], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
