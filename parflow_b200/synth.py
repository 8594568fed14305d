"""Seeded synthetic inputs for the Richards workloads.

No public dataset backs these workloads; every field is generated here from a
seed so that the reference CPU build, the oracle and the CUDA library all see
identical bits (the reference reads them back as PFB files).

* ``lognormal_field``: Gaussian field with exponential covariance
  exp(-|r/L|) (anisotropic correlation lengths in cells) by FFT spectral
  synthesis on a zero-padded periodic box, normalised to mean 0 / std 1.
* ``smoothed_slopes``: smoothed Gaussian field mapped to sign * [lo, hi] for
  topographic slopes.
"""

from __future__ import annotations

import numpy as np


def _spectral_exponential(shape, corr, rng):
    """Real Gaussian field on ``shape`` (z, y, x) with exponential covariance."""
    pads = [int(min(2 * n, n + 4 * max(1, int(np.ceil(c))))) for n, c in zip(shape, corr)]
    ks = []
    for n, c in zip(pads, corr):
        k = np.fft.fftfreq(n) * 2.0 * np.pi * float(c)
        ks.append(k)
    kz, ky, kx = np.meshgrid(ks[0], ks[1], np.fft.rfftfreq(pads[2]) * 2.0 * np.pi * float(corr[2]),
                             indexing="ij")
    k2 = kz * kz + ky * ky + kx * kx
    # 3D exponential covariance spectrum ~ (1 + |kL|^2)^-2
    amp = 1.0 / (1.0 + k2)
    noise = rng.standard_normal(pads)
    spec = np.fft.rfftn(noise) * amp
    field = np.fft.irfftn(spec, s=pads, axes=(0, 1, 2))
    return field[: shape[0], : shape[1], : shape[2]]


def lognormal_field(shape, corr, seed: int, sigma: float = 1.0, mean: float = 0.0):
    """Return g with mean 0 / std 1 (then scaled: mean + sigma * g)."""
    rng = np.random.default_rng(seed)
    g = _spectral_exponential(tuple(shape), tuple(corr), rng)
    g = (g - g.mean()) / g.std()
    return mean + sigma * g


def smoothed_slopes(shape2d, seed: int, lo: float, hi: float, corr: float = 8.0):
    """Slopes with magnitude in [lo, hi] and random sign from a smooth field."""
    rng = np.random.default_rng(seed)
    g = _spectral_exponential((1,) + tuple(shape2d), (1.0, corr, corr), rng)[0]
    g = (g - g.mean()) / g.std()
    mag = lo + (hi - lo) * np.clip(np.abs(g) / 3.0, 0.0, 1.0)
    return np.where(g >= 0.0, mag, -mag)


__all__ = ["lognormal_field", "smoothed_slopes"]
