"""pytest configuration: the `gpu` marker and shared fixtures.

CPU tests (-m "not gpu") exercise the oracle against the reference's own CPU
code and known-answer tests, and check that librmcuda.so loads and exports its
ABI.  GPU tests (-m gpu) run the CUDA path through the C ABI and compare it
with the oracle.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build_oracle()
    return pyoracle


@pytest.fixture(scope="session")
def ref(oracle):
    """The reference's own CPU engine (scene/bvh/camera), or skip if it was never built."""
    oracle.build_ref()
    lib = oracle.ref_lib()
    if lib is None:
        pytest.skip("oracle/_ref/libref.so not built (needs the reference checkout)")
    return lib


@pytest.fixture(scope="session")
def backend():
    import raymotion_b200 as rb
    from raymotion_b200 import build
    if not build.LIB.exists():
        build.build()
    return rb.Backend(0)


@pytest.fixture(autouse=True)
def _clean_env(monkeypatch):
    for k in ("UOW2_NOADAPT", "UOW2_NOMIS", "RAYMOTION_RESTIR", "RAYMOTION_RESTIR_CANDIDATES",
              "RAYMOTION_RESTIR_SPATIAL", "RAYMOTION_RESTIR_TEMPORAL", "RAYMOTION_DENOISE"):
        monkeypatch.delenv(k, raising=False)
