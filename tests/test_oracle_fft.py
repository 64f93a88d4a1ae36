"""The oracle's FFT against numpy's pocketfft (stand-in for FFTW3)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "fft_golden.npz")


def test_fft_golden_vectors():
    z = np.load(GOLD)
    keys = sorted(k[2:] for k in z.files if k.startswith("x_"))
    assert keys
    for key in keys:
        nx, ny, nz = (int(v) for v in key.split("_"))
        g = O.Grid(nx, ny, nz)
        X = O.fft2_r2c(g, z["x_" + key])
        assert np.linalg.norm(X - z["X_" + key]) <= 1e-14 * np.linalg.norm(z["X_" + key]), key
        y = O.fft2_c2r(g, z["X_" + key])
        assert np.linalg.norm(y - z["y_" + key]) <= 1e-14 * np.linalg.norm(z["y_" + key]), key


@pytest.mark.parametrize("nx,nz", [(64, 64), (256, 128), (512, 8), (96, 112), (80, 48), (14, 21)])
def test_fft_against_numpy(nx, nz):
    g = O.Grid(nx, 2, nz)
    x = np.random.default_rng(nx * 1000 + nz).standard_normal((2, nz, nx))
    X = O.fft2_r2c(g, x)
    ref = np.fft.rfft2(x, axes=(1, 2))
    assert np.linalg.norm(X - ref) <= 1e-14 * np.linalg.norm(ref)
    y = O.fft2_c2r(g, X)
    assert np.abs(y / (nx * nz) - x).max() < 1e-13
