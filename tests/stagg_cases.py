"""Closed forms and recipes of the staggered sixth-order scheme (cd06stagg),
shared by the oracle test and the GPU test.

* Periodic lines: a Fourier mode goes to its staggered modified wavenumber /
  transfer function times the mode at the output points (cells at
  (j + 1/2) dz, edges at j dz): first derivative 2 (a sin(w/2) + b sin(3w/2))
  / ((1 + 2 alpha cos w) dz) with a = 63/62, b = 17/186, alpha = 9/62
  (cd06stagg.F90:174, 307); interpolation (2 a cos(w/2) + 2 b cos(3w/2)) /
  (1 + 2 alpha cos w) with a = 3/4, b = 1/20, alpha = 3/10 (:176, 532); second
  derivative -(2 a (cos w - 1) + 2 b (cos 2w - 1)) / ((1 + 2 alpha cos w) dz^2)
  with a = 12/11, b = 3/44, alpha = 2/11 (:175, 411).
* Non-periodic lines with even / odd closures: a mode with that parity about
  both boundary edges (cos or sin of 3z on [0, pi] or [0, pi/2]) is
  reproduced exactly, its mirror image being the mode itself; the C2C / E2E
  first derivatives use the cd06 wavenumber (a = 7/9, b = 1/36, alpha = 1/3).
* One-sided closures reproduce polynomials up to their order: 3 for the first
  derivatives E2C / C2E and the E2C interpolation, 4 for the C2C first
  derivative, 2 for the C2E interpolation (measured on the oracle; a wrong
  closure coefficient breaks them).
* tests/test_STAGGcd06.F90: periodic, nz = 8 on [0, 1], f = sin(2 pi z) +
  i cos(2 pi z) on edges and cells; ddz_E2C, ddz_C2E, d2dz2_C2C, d2dz2_E2E,
  InterpZ_E2C, InterpZ_C2E against the exact functions.
"""
from __future__ import annotations

import itertools

import numpy as np

OPS = ["ddz_E2C", "ddz_C2E", "ddz_C2C", "ddz_E2E", "d2dz2_C2C", "d2dz2_E2E", "InterpZ_E2C", "InterpZ_C2E"]
SIDED_ORDER = {"ddz_E2C": 3, "ddz_C2E": 3, "ddz_C2C": 4, "InterpZ_E2C": 3, "InterpZ_C2E": 2}


def kd1(w, dz):
    a, b, al = 63 / 62, (17 / 62) / 3, 9 / 62
    return 2 * (a * np.sin(w / 2) + b * np.sin(3 * w / 2)) / ((1 + 2 * al * np.cos(w)) * dz)


def kd1c(w, dz):
    a, b, al = (14 / 9) / 2, (1 / 9) / 4, 1 / 3
    return 2 * (a * np.sin(w) + b * np.sin(2 * w)) / ((1 + 2 * al * np.cos(w)) * dz)


def tint(w):
    a, b, al = 0.75, 0.05, 0.3
    return (2 * a * np.cos(w / 2) + 2 * b * np.cos(3 * w / 2)) / (1 + 2 * al * np.cos(w))


def kd2(w, dz):
    a, b, al = 12 / 11, (3 / 11) / 4, 2 / 11
    return -(2 * a * (np.cos(w) - 1) + 2 * b * (np.cos(2 * w) - 1)) / ((1 + 2 * al * np.cos(w)) * dz ** 2)


def grids(n, dz):
    return np.arange(n + 1) * dz, (np.arange(n) + 0.5) * dz


def periodic_cases(n, kmax=None):
    """(name, f planes, expected planes, m) for modes m = 1..kmax on [0, 1)."""
    dz = 1.0 / n
    zE, zC = grids(n, dz)
    out = []
    for m in range(1, (kmax or n // 2 - 1) + 1):
        k = 2 * np.pi * m
        w = k * dz
        s = lambda z: np.sin(k * z + 0.3)  # noqa: E731
        c = lambda z: np.cos(k * z + 0.3)  # noqa: E731
        out += [("ddz_E2C", s(zE), kd1(w, dz) * c(zC), m), ("ddz_C2E", s(zC), kd1(w, dz) * c(zE), m),
                ("InterpZ_E2C", s(zE), tint(w) * s(zC), m), ("InterpZ_C2E", s(zC), tint(w) * s(zE), m),
                ("d2dz2_C2C", s(zC), -kd2(w, dz) * s(zC), m), ("d2dz2_E2E", s(zE), -kd2(w, dz) * s(zE), m)]
    return out


def parity_cases(n):
    """(bot_even, top_even, name, f, expected) for every even / odd pair."""
    out = []
    for be, te in itertools.product((True, False), repeat=2):
        L = np.pi if be == te else np.pi / 2
        k = 3.0
        dz = L / n
        zE, zC = grids(n, dz)
        f0, f1 = (np.cos, lambda x: -np.sin(x)) if be else (np.sin, np.cos)
        w = k * dz
        out += [(be, te, dz, "ddz_E2C", f0(k * zE), kd1(w, dz) * f1(k * zC)),
                (be, te, dz, "ddz_C2E", f0(k * zC), kd1(w, dz) * f1(k * zE)),
                (be, te, dz, "ddz_C2C", f0(k * zC), kd1c(w, dz) * f1(k * zC)),
                (be, te, dz, "ddz_E2E", f0(k * zE), kd1c(w, dz) * f1(k * zE)),
                (be, te, dz, "InterpZ_E2C", f0(k * zE), tint(w) * f0(k * zC)),
                (be, te, dz, "InterpZ_C2E", f0(k * zC), tint(w) * f0(k * zE)),
                (be, te, dz, "d2dz2_C2C", f0(k * zC), -kd2(w, dz) * f0(k * zC)),
                (be, te, dz, "d2dz2_E2E", f0(k * zE), -kd2(w, dz) * f0(k * zE))]
    return out


def sided_cases(n, seed=0):
    """(name, dz, f, expected) with polynomials of each sided closure's order on [0, 1]."""
    dz = 1.0 / n
    zE, zC = grids(n, dz)
    rng = np.random.default_rng(seed)
    out = []
    for name, d in SIDED_ORDER.items():
        P = np.polynomial.Polynomial(rng.uniform(0.5, 1.0, d + 1))
        dP = P.deriv()
        src, dst = (zE, zC) if name.endswith("E2C") else ((zC, zE) if name.endswith("C2E") else (zC, zC))
        ex = dP(dst) if name.startswith("ddz") else P(dst)
        out.append((name, dz, P(src), ex))
    return out


def reference_recipe():
    """tests/test_STAGGcd06.F90:13-76: (name, f, exact) on nz = 8, complex."""
    nz = 8
    dz = 1.0 / nz
    zE = np.arange(nz + 1) * dz
    zC = 0.5 * (zE[1:] + zE[:-1])
    tp = 2 * np.pi
    fE = np.sin(tp * zE) + 1j * np.cos(tp * zE)
    fC = np.sin(tp * zC) + 1j * np.cos(tp * zC)
    dfE = tp * np.cos(tp * zE) + 1j * (-tp * np.sin(tp * zE))
    dfC = tp * np.cos(tp * zC) + 1j * (-tp * np.sin(tp * zC))
    d2fE = -(tp ** 2) * np.sin(tp * zE) + 1j * (-(tp ** 2)) * np.cos(tp * zE)
    d2fC = -(tp ** 2) * np.sin(tp * zC) + 1j * (-(tp ** 2)) * np.cos(tp * zC)
    return nz, dz, [("ddz_E2C", fE, dfC), ("ddz_C2E", fC, dfE), ("d2dz2_C2C", fC, d2fC), ("d2dz2_E2E", fE, d2fE),
                    ("InterpZ_E2C", fE, fC), ("InterpZ_C2E", fC, fE)]


def cplx_apply(S, name, f):
    """The oracle's operator on a complex line: real and imaginary parts alone."""
    re = S.apply(name, np.ascontiguousarray(f.real)[:, None, None])[:, 0, 0]
    im = S.apply(name, np.ascontiguousarray(f.imag)[:, None, None])[:, 0, 0]
    return re + 1j * im
