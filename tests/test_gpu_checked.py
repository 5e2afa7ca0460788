"""The bounds-checked build (librmcuda_checked.so, RMCUDA_CHECKED) on the GPU.

Every index the kernels read from a device structure is compared with its
array there; a bad one sets an error bit and the call fails instead of
reading out of bounds.  This runs parity tests of the plain path, the ReSTIR
chain (wavefront with its tail, and the megakernel), the batch, the device
BVH and the no-alloc ray queries with RAYMOTION_CUDA_CHECKED=1, in a child
process that loads the checked library: they pass unchanged, so no check fires
on them and the checked kernels give the same results bit for bit.
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu


def test_parity_suite_passes_with_bounds_checks():
    from raymotion_b200 import build
    if not build.LIB_CHECKED.exists():
        build.build(checked=True)
    env = dict(os.environ, RAYMOTION_CUDA_CHECKED="1")
    sel = ("cornell_plain_path or closest_hit_ids or restir_chain_matches_oracle or wavefront_shading_variants or "
           "batch_equals_single_image or batch_of_one_cornell or device_builders or refit_and_rebuild or "
           "wide_bvh_hits or trace_noalloc_matches")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu", "-k", sel,
                        "tests/test_gpu_parity.py", "tests/test_gpu_batch.py", "tests/test_gpu_bvh.py",
                        "tests/test_zz_no_alloc.py"],
                       capture_output=True, text=True, env=env, cwd=ROOT, timeout=1800)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "failed" not in r.stdout
