"""include/rm_detmath.h against double-precision libm (CPU)."""
import numpy as np


def _ulps(a32, ref64):
    ref32 = ref64.astype(np.float32)
    spacing = np.spacing(np.abs(ref32)).astype(np.float64)
    return np.abs(a32.astype(np.float64) - ref64) / np.maximum(spacing, np.finfo(np.float32).tiny)


def test_sincos_on_sampling_range(oracle):
    # azimuths are u * 2pi with u in [0, 1) (pathtrace.metal:208, :227)
    u = np.linspace(0, 1, 200001, endpoint=False, dtype=np.float32)
    phi = (u * np.float32(2 * np.pi)).astype(np.float32)
    s, c = oracle.detmath(0, phi)
    x = phi.astype(np.float64)
    assert np.max(np.abs(s - np.sin(x))) < 4e-7
    assert np.max(np.abs(c - np.cos(x))) < 4e-7
    big = np.abs(np.sin(x)) > 1e-3
    assert np.max(_ulps(s[big], np.sin(x[big]))) <= 4


def test_sincos_wider_arguments(oracle):
    x = np.linspace(-200, 200, 100001, dtype=np.float32)
    s, c = oracle.detmath(0, x)
    assert np.max(np.abs(s - np.sin(x.astype(np.float64)))) < 1e-6
    assert np.max(np.abs(c - np.cos(x.astype(np.float64)))) < 1e-6


def test_atan(oracle):
    x = np.concatenate([np.linspace(-50, 50, 100001), np.array([np.inf, -np.inf, 0.0, 1e-30, 1e30])]).astype(
        np.float32)
    y, _ = oracle.detmath(1, x)
    assert np.max(_ulps(y[np.abs(y) > 1e-30], np.arctan(x.astype(np.float64))[np.abs(y) > 1e-30])) <= 4
    assert y[-5] == np.float32(np.pi / 2) and y[-4] == -np.float32(np.pi / 2)


def test_exp(oracle):
    x = np.linspace(-87, 88, 200001, dtype=np.float32)
    y, _ = oracle.detmath(2, x)
    assert np.max(_ulps(y, np.exp(x.astype(np.float64)))) <= 4
    z, _ = oracle.detmath(2, np.array([-200.0, 100.0, -0.0], np.float32))
    assert z[0] == 0 and np.isinf(z[1]) and z[2] == 1
