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


def test_sequence_reference_is_reproduced(oracle):
    """The animated sequence's frame-33 reference (relmse_sequence33.npz):
    64 of its pixels at 512 spp with another seed."""
    g = np.load(GOLDEN / "relmse_sequence33.npz")
    assert int(g["spp"]) == 16384 and len(g["pixels"]) == 4096
    scene, cam, cfg = workloads()["sequence33"]()
    assert scene.n_tris == 1_158_148
    scene = oracle.with_reference_bvh(scene)
    pix, ref = g["pixels"][::64], g["ref"][::64]
    cfg.spp = 512
    a = oracle.render_f64(scene, cam, cfg, 7, pixels=pix)
    assert (ref > 0).mean() > 0.2
    assert np.mean((a - ref) ** 2 / (ref ** 2 + 0.01)) < 0.1


def test_batch_references_cover_the_workload_and_are_reproduced(oracle):
    """relmse_batch.npz holds 256 pixels of each of the 64 batched scenes;
    two small scenes' references are reproduced at 512 spp."""
    from raymotion_b200.scenes import batch_workload, sized_field
    g = np.load(GOLDEN / "relmse_batch.npz")
    specs = batch_workload(seed=3, n_scenes=64)
    assert sorted(set(g["scene"].tolist())) == list(range(64))
    for k in sorted(range(64), key=lambda i: specs[i]["n_tris"])[:2]:
        sel = g["scene"] == k
        assert sel.sum() == 256
        sb, cam, cfg = sized_field(**specs[k])
        assert g["pixels"][sel].max() < cfg.width * cfg.height
        scene = oracle.with_reference_bvh(sb.pack())
        cfg.spp = 512
        a = oracle.render_f64(scene, cam, cfg, 11, pixels=g["pixels"][sel])
        ref = g["ref"][sel]
        assert np.mean((a - ref) ** 2 / (ref ** 2 + 0.01)) < 0.1, k
