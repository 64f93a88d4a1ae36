"""Generate tests/golden/fft_golden.npz: FFT fixtures for the oracle.

The reference's FFT is FFTW3 (not vendored, not installed here; README.md:11
asks for fftw >= 3.1), called as a batched rank-2 r2c/c2r over [nz, nx] per
y plane with the forward sign and no normalisation
(src/modules/pressure/pressure_backend_fftw.f90:22-49).  numpy's pocketfft
computes the same transform (numpy.fft.rfft2 over the last two axes), so its
outputs on seeded inputs pin the oracle's own FFT at that boundary.

Run:  python tests/golden/make_fft_golden.py
"""
import os

import numpy as np

CASES = [(8, 3, 6), (24, 2, 18), (64, 1, 32), (48, 1, 40), (200, 1, 10), (30, 2, 14)]


def main():
    out = {}
    rng = np.random.default_rng(20261203)
    for nx, ny, nz in CASES:
        x = rng.standard_normal((ny, nz, nx))
        X = np.fft.rfft2(x, axes=(1, 2))
        y = np.fft.irfft2(X, s=(nz, nx), axes=(1, 2)) * (nx * nz)
        key = f"{nx}_{ny}_{nz}"
        out["x_" + key] = x
        out["X_" + key] = X
        out["y_" + key] = y
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fft_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
