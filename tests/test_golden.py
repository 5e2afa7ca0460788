"""The committed FP64 references of the relMSE checks (tests/golden/make_relmse_refs.py)
are reproduced by an independent oracle run: 128 of their pixels at 512 spp with
another seed agree within the noise of 512 spp."""
import numpy as np
import pytest

from tests.golden.make_relmse_refs import workloads

GOLDEN = __import__("pathlib").Path(__file__).with_name("golden")


@pytest.mark.parametrize("name", ["cornell", "icosphere720"])
def test_relmse_reference_is_reproduced(oracle, name):
    g = np.load(GOLDEN / f"relmse_{name}.npz")
    assert int(g["spp"]) == 16384 and len(g["pixels"]) == 4096
    scene, cam, cfg = workloads()[name]()
    scene = oracle.with_reference_bvh(scene)
    pix = g["pixels"][::32]
    ref = g["ref"][::32]
    cfg.spp = 512
    a = oracle.render_f64(scene, cam, cfg, 7, pixels=pix)
    live = ref > 0
    assert live.mean() > 0.2
    # relMSE of 512 spp against the converged reference: noise-sized (well under 1e-1)
    # and the mean radiance of the pixels agrees within a few per cent
    rel = np.mean((a - ref) ** 2 / (ref ** 2 + 0.01))
    assert rel < 0.1, rel
    assert abs(a[live].sum() / ref[live].sum() - 1.0) < 0.05
