"""Seeded synthetic coefficient fields of the benchmark configurations.

  lognormal_modes  diffusion kappa = exp(g), g a Gaussian random field with
                   mean 0, standard deviation sigma and squared-exponential
                   correlation of length ell, as a sum of random-phase Fourier
                   modes (spectral sampling); used with PMG_COEF_LOGNORMAL
  curl_modes       convection b = curl psi of an 8-mode Fourier vector
                   potential, scaled so that max|b| = bmax; PMG_COEF_CURL_FOURIER
Each mode row is (kx, ky, kz, amplitude, phase, ax, ay, az).
"""
import numpy as np


def lognormal_modes(seed, n_modes=64, ell=0.1, sigma=1.0):
    rng = np.random.default_rng(seed)
    m = np.zeros((n_modes, 8))
    m[:, 0:3] = rng.normal(scale=1.0 / (2 * np.pi * ell), size=(n_modes, 3))
    m[:, 3] = sigma * np.sqrt(2.0 / n_modes)
    m[:, 4] = rng.uniform(0, 2 * np.pi, n_modes)
    return m


def curl_modes(seed, n_modes=8, bmax=None):
    """Modes and the scale factor that makes max|b| = bmax (bmax log-uniform in [1, 100] if None)."""
    rng = np.random.default_rng(seed)
    m = np.zeros((n_modes, 8))
    m[:, 0:3] = rng.integers(-2, 3, size=(n_modes, 3))
    m[m[:, 0:3].sum(axis=1) == 0, 0] = 1
    m[:, 3] = rng.normal(size=n_modes) / np.sqrt(n_modes)
    m[:, 4] = rng.uniform(0, 2 * np.pi, n_modes)
    m[:, 5:8] = rng.normal(size=(n_modes, 3))
    if bmax is None:
        bmax = float(np.exp(rng.uniform(0.0, np.log(100.0))))
    g = np.linspace(0, 1, 17)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    bx = np.zeros_like(X); by = np.zeros_like(X); bz = np.zeros_like(X)
    for M in m:
        arg = 2 * np.pi * (M[0] * X + M[1] * Y + M[2] * Z) + M[4]
        s = -M[3] * np.sin(arg) * 2 * np.pi
        gx, gy, gz = s * M[0], s * M[1], s * M[2]
        bx += gy * M[7] - gz * M[6]
        by += gz * M[5] - gx * M[7]
        bz += gx * M[6] - gy * M[5]
    peak = float(np.sqrt(bx ** 2 + by ** 2 + bz ** 2).max())
    return m, bmax / max(peak, 1e-12)
