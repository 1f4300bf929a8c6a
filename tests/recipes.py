"""Closed forms and test recipes of the reference, restated for the oracle tests.

* ``mod_wavenumber``: the modified wavenumbers / transfer function of
  src/utilities/spectral.F90:938-1010 (GetCF90TransferFunction,
  GetCD10ModWaveNum, GetCD10D2ModWaveNum, GetCD06ModWaveNum).
* ``recipe_errors``: the set-ups of the reference tests tests/test_cd06.F90,
  test_cd10_NP.F90, test_cd10_der2.F90 and test_cf90.F90 (grid, function,
  closures), evaluated through the oracle.
"""
import numpy as np

import oracle


def _cd10_consts():
    # cd10.F90:16-30: alpha/beta/a/b/c for the first and second derivatives
    a1, b1 = 1.0 / 2.0, 1.0 / 20.0
    d1 = dict(alpha=a1, beta=b1, a=(17.0 / 12.0) / 2.0, b=(101.0 / 150.0) / 4.0, c=(1.0 / 100.0) / 6.0)
    a2, b2 = 334.0 / 899.0, 43.0 / 1798.0
    d2 = dict(alpha=a2, beta=b2, a=(1065.0 / 1798.0) / 1.0, b=(1038.0 / 899.0) / 4.0, c=(79.0 / 1798.0) / 9.0)
    return d1, d2


def mod_wavenumber(scheme, kind, k, dx):
    """D e^{ikx} = (i k') e^{ikx} (first derivative), -(k'') e^{ikx} (second),
    T e^{ikx} (filter); returns k', k'' or T."""
    w = k * dx
    if scheme == oracle.CD06:  # spectral.F90:987-1010
        alpha = 1.0 / 3.0
        a, b = (2.0 / 9.0) * (8 - 3 * alpha), (1.0 / 18.0) * (-17 + 57 * alpha)
        return (a * np.sin(w) + (b / 2) * np.sin(2 * w)) / (1 + 2 * alpha * np.cos(w)) / dx
    d1, d2 = _cd10_consts()
    if scheme == oracle.CD10 and kind == oracle.D1:  # spectral.F90:950-961
        c = d1
        num = 2 * c["a"] * np.sin(w) + 2 * c["b"] * np.sin(2 * w) + 2 * c["c"] * np.sin(3 * w)
        return num / (1 + 2 * c["alpha"] * np.cos(w) + 2 * c["beta"] * np.cos(2 * w)) / dx
    if scheme == oracle.CD10:  # spectral.F90:965-984 (which returns this times dx)
        c = d2
        a, b, cc = c["a"], c["b"] * 4, c["c"] * 9
        num = 2 * a * (1 - np.cos(w)) + (b / 2) * (1 - np.cos(2 * w)) + (2 * cc / 9) * (1 - np.cos(3 * w))
        return num / (1 + 2 * c["alpha"] * np.cos(w) + 2 * c["beta"] * np.cos(2 * w)) / dx ** 2
    # cf90 transfer function, spectral.F90:938-948 (cf90.F90:16-48 constants)
    alpha, beta = 6.6624e-1, 1.6688e-1
    a, b, c, d, e = 9.9965e-1, 6.6652e-1, 1.6674e-1, 4.0e-5, -5.0e-6
    num = a + 2 * b * np.cos(w) + 2 * c * np.cos(2 * w) + 2 * d * np.cos(3 * w) + 2 * e * np.cos(4 * w)
    return num / (1 + 2 * alpha * np.cos(w) + 2 * beta * np.cos(2 * w))



def recipe_errors() -> dict:
    """Max |D f - exact| of the reference tests' recipes, through the oracle."""
    out = {}
    # tests/test_cd06.F90: periodic, sin(omega x), omega = 1 (x on 256 points; y, z short here)
    n = 256
    dx = 2 * np.pi / n
    x = np.arange(n) * dx
    f = np.broadcast_to(np.sin(x)[None, None, :], (2, 3, n)).copy()
    o = oracle.OracleOp(oracle.CD06, n, dx, True)
    out["cd06_periodic_dd1"] = float(np.abs(o.apply(oracle.D1, 1, f, 3, 2).reshape(f.shape) - np.cos(x)).max())
    # tests/test_cd10_NP.F90: bounded, dx = pi/2/(n-1), cos x cos y cos z, closures (1, -1)
    n = 32
    dx = np.pi / 2 / (n - 1)
    x = np.arange(n) * dx
    f1 = np.cos(x)
    f = np.broadcast_to(f1[None, None, :], (2, 3, n)).copy()
    o = oracle.OracleOp(oracle.CD10, n, dx, False)
    out["cd10_np_dd1"] = float(np.abs(o.apply(oracle.D1, 1, f, 3, 2, 1, -1).reshape(f.shape) + np.sin(x)).max())
    out["cd10_np_d2d1"] = float(np.abs(o.apply(oracle.D2, 1, f, 3, 2, 1, -1).reshape(f.shape) + np.cos(x)).max())
    # tests/test_cd10_der2.F90: periodic, 32 points, second derivative of sin x
    n = 32
    dx = 2 * np.pi / n
    x = np.arange(n) * dx
    f = np.broadcast_to(np.sin(x)[None, None, :], (1, 1, n)).copy()
    o = oracle.OracleOp(oracle.CD10, n, dx, True)
    out["cd10_der2"] = float(np.abs(o.apply(oracle.D2, 1, f, 1, 1).reshape(f.shape) + np.sin(x)).max())
    # tests/test_cf90.F90: periodic, omega = 12, f = cos(w x), filtered = T(w dx) f
    n, w = 32, 12.0
    dx = 2 * np.pi / n
    x = np.arange(n) * dx
    f = np.broadcast_to(np.cos(w * x)[None, None, :], (2, 2, n)).copy()
    o = oracle.OracleOp(oracle.CF90, n, 1.0, True)
    tf = mod_wavenumber(oracle.CF90, oracle.FILTER, w, dx)
    out["cf90_tf"] = float(np.abs(o.apply(oracle.FILTER, 1, f, 2, 2).reshape(f.shape) - tf * np.cos(w * x)).max())
    return out
