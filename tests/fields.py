"""Seeded synthetic fields with the shapes and spectra of the benchmark
configurations (the reference measures on solver fields; these stand in).

Arrays are C-ordered (n3, n2, n1) numpy float64 arrays, i.e. the column-major
field f(n1, n2, n3) of the reference.
"""
from __future__ import annotations

import numpy as np


def sinusoids(n: int, seed: int, modes: int = 8, kmax: int = 16) -> np.ndarray:
    """Sum of `modes` plane waves sin(kx x + ky y + kz z + phi) on [0, 2pi)^3,
    integer wavenumbers uniform in 1..kmax, phases uniform in [0, 2pi)."""
    rng = np.random.default_rng(seed)
    x = np.arange(n) * (2 * np.pi / n)
    f = np.zeros((n, n, n))
    for _ in range(modes):
        kx, ky, kz = rng.integers(1, kmax + 1, size=3)
        ph = rng.uniform(0, 2 * np.pi)
        f += np.sin(kz * x[:, None, None] + ky * x[None, :, None] + kx * x[None, None, :] + ph)
    return f


def spectrum53(shape: tuple[int, int, int], seed: int, kfrac: float = 2.0 / 3.0) -> np.ndarray:
    """Random-phase Fourier synthesis with |u(k)|^2 ~ |k|^(-5/3) for
    1 <= |k| <= kfrac * n/2, zero mean, unit RMS.  shape = (n3, n2, n1)."""
    rng = np.random.default_rng(seed)
    n3, n2, n1 = shape
    k3 = np.fft.fftfreq(n3, 1.0 / n3)[:, None, None]
    k2 = np.fft.fftfreq(n2, 1.0 / n2)[None, :, None]
    k1 = np.fft.rfftfreq(n1, 1.0 / n1)[None, None, :]
    kk = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2)
    kmax = kfrac * min(shape) / 2
    amp = np.where((kk >= 1) & (kk <= kmax), np.power(np.maximum(kk, 1.0), -5.0 / 6.0) / np.maximum(kk, 1.0), 0.0)
    ph = rng.uniform(0, 2 * np.pi, size=amp.shape)
    spec = amp * np.exp(1j * ph)
    f = np.fft.irfftn(spec, s=shape, axes=(0, 1, 2))
    f -= f.mean()
    rms = np.sqrt(np.mean(f * f))
    return f / rms if rms > 0 else f


def poly_z(shape: tuple[int, int, int], seed: int) -> np.ndarray:
    """3rd-order polynomial in z (seeded coefficients in [-1,1]) plus 0.1 sin of
    seeded wavenumbers 1..32 in x and y; z in [0,1] (dz = 1/(n3-1))."""
    rng = np.random.default_rng(seed)
    n3, n2, n1 = shape
    c = rng.uniform(-1, 1, size=4)
    kx, ky = rng.integers(1, 33, size=2)
    z = np.linspace(0.0, 1.0, n3)[:, None, None]
    x = (np.arange(n1) * (2 * np.pi / n1))[None, None, :]
    y = (np.arange(n2) * (2 * np.pi / n2))[None, :, None]
    return (c[0] + c[1] * z + c[2] * z ** 2 + c[3] * z ** 3) + 0.1 * np.sin(kx * x + ky * y)


def na_nb(shape: tuple[int, int, int], axis: int) -> tuple[int, int]:
    n3, n2, n1 = shape
    return {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]


def line_len(shape: tuple[int, int, int], axis: int) -> int:
    n3, n2, n1 = shape
    return {1: n1, 2: n2, 3: n3}[axis]


def rel_err(x: np.ndarray, r: np.ndarray) -> float:
    """max|x - r| / max|r| (the parity metric)."""
    den = float(np.abs(r).max())
    return float(np.abs(x - r).max()) / (den if den > 0 else 1.0)
