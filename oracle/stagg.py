"""Staggered sixth-order compact scheme (TEST INFRASTRUCTURE ONLY).

A numpy restatement of the reference module ``cd06staggstuff``
(src/derivatives/cd06stagg.F90 and the STAGG_CD06_files/*.F90 it includes):
first derivatives edge->cell (E2C), cell->edge (C2E), cell->cell (C2C) and
edge->edge (E2E), second derivatives C2C and E2E, and interpolation E2C and
C2E, along z of (n1, n2, nz) fields, periodic (cyclic LU) or non-periodic
(Thomas, with even / odd symmetric or one-sided closures).  Each array
statement of the reference is restated on whole z planes, in the same order
and with the same grouping, so every element is computed as the reference
computes it.  The cell grid has n points, the edge grid nE = n + 1.

Fields are numpy float64 arrays of shape (nz, n2, n1) (C order: the
reference's column-major f(n1, n2, nz)).  A complex field is its real and
imaginary parts filtered alone (the coefficients are real), so it is the real
operator on the interleaved (nz, n2, 2*n1) view.

Only ``tests/`` use this module; the product never imports it.
"""
from __future__ import annotations

import numpy as np

E2C, C2E, C2C, E2E = "E2C", "C2E", "C2C", "E2E"

# cd06stagg.F90:18-57 (edge-node closures of the C2C first derivative, Lele)
_alpha, _p, _q, _r, _s = 3.0, 17.0 / 6.0, 3.0 / 2.0, 3.0 / 2.0, -1.0 / 6.0
_alpha06d1 = 1.0 / 3.0
_a06d1 = (14.0 / 9.0) / 2.0
_b06d1 = (1.0 / 9.0) / 4.0
_qhat, _rhat, _alpha_hat = _a06d1, _b06d1, _alpha06d1
_q_p, _alpha_p = 3.0 / 4.0, 1.0 / 4.0
_alpha_pp = (((40 * _alpha_hat - 1) * _q + 7 * (4 * _alpha_hat - 1) * _s)
             / (16 * (_alpha_hat + 2) * _q + 8 * (1 - 4 * _alpha_hat) * _s))
_q_pp = (1.0 / 3.0) * (_alpha_pp + 2)
_r_pp = (1.0 / 12.0) * (4 * _alpha_pp - 1)
_w1 = (2 * _alpha_hat + 1) / (2 * (_q + _s))
_w2 = ((8 * _alpha_hat + 7) * _q - 6 * (2 * _alpha_hat + 1) * _r + (8 * _alpha_hat + 7) * _s) / (9 * (_q + _s))
_w3 = (4 * (_alpha_hat + 2) * _q + 2 * (1 - 4 * _alpha_hat) * _s) / (9 * (_q + _s))
_w0s, _w1s = 223.0 / 186.0, 61.0 / 62.0


def _cyclic_lu(n: int, b: float, d: float, a: float) -> np.ndarray:
    """ComputeLU (cd06stagg.F90:631-672): columns bc, h, 1/c, a/c, v/c (0-based: 0..4)."""
    LU = np.zeros((n, 5))
    bc, h, c, aa, v = (LU[:, k] for k in range(5))
    c[0] = d
    v[0] = b
    h[0] = a / c[0]
    for i in range(1, n - 1):
        c[i] = d - (b / c[i - 1]) * a
    for i in range(1, n - 2):
        v[i] = -(b / c[i - 1]) * v[i - 1]
        h[i] = -(a / c[i]) * h[i - 1]
    v[n - 2] = a - (b / c[n - 3]) * v[n - 3]
    h[n - 2] = (b - h[n - 3] * a) / c[n - 2]
    acc = 0.0
    for i in range(n - 1):  # SUM(h(1:n-1)*v(1:n-1)) in index order
        acc += h[i] * v[i]
    c[n - 1] = d - acc
    bc[1 : n - 1] = b / c[: n - 2]
    aa[: n - 2] = a
    c[:] = 1.0 / c
    aa[:] = aa * c
    v[:] = v * c
    return LU


def _thomas(ddn, dg, dup) -> np.ndarray:
    """ComputeTri_common.F90: columns ddn*den, den, cp."""
    n = len(dg)
    cp = np.zeros(n)
    den = np.zeros(n)
    cp[0] = dup[0] / dg[0]
    for i in range(1, n - 1):
        cp[i] = dup[i] / (dg[i] - ddn[i] * cp[i - 1])
    den[0] = 1.0 / dg[0]
    den[1:] = 1.0 / (dg[1:] - ddn[1:] * cp[: n - 1])
    return np.stack([ddn * den, den, cp], axis=1)


class Stagg:
    """cd06stagg: init_periodic(nx, dx) or init_nonperiodic(nx, dx, isTopEven,
    isBotEven, isTopSided, isBotSided) (cd06stagg.F90:170-232)."""

    def __init__(self, n: int, dx: float, periodic: bool = True, top_even: bool = True, bot_even: bool = True,
                 top_sided: bool = False, bot_sided: bool = False):
        if n <= 4:
            raise ValueError("CD06_stagg requires at least 4 points (GracefulExit 21)")
        self.n, self.nE, self.dx = n, n + 1, dx
        self.onebydx = 1.0 / dx
        self.onebydx2 = self.onebydx / dx
        self.periodic = periodic
        self.top_even, self.bot_even = top_even, bot_even
        self.top_sided, self.bot_sided = top_sided, bot_sided
        if periodic:
            self.LU_D1 = _cyclic_lu(n, 9.0 / 62.0, 1.0, 9.0 / 62.0)
            self.LU_D2 = _cyclic_lu(n, 2.0 / 11.0, 1.0, 2.0 / 11.0)
            self.LU_interp = _cyclic_lu(n, 3.0 / 10.0, 1.0, 3.0 / 10.0)
        else:
            self.tri = {k: getattr(self, "_tri_" + k)() for k in
                        ("d1_e2c", "d1_c2e", "d1_c2c", "d1_e2e", "d2_e2e", "d2_c2c", "interp_c2e", "interp_e2c")}

    # ---- Thomas factors, ComputeTri_allRoutines.F90 ---------------------------------------
    def _tri_d1_e2c(self):  # :1-50
        n, alpha, alpha1, alpha0 = self.n, 9.0 / 62.0, 37.0 / 183.0, -1.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        if self.top_sided:
            ddn[n - 1] = _w0s * alpha0; dg[n - 1] = _w0s
            ddn[n - 2] = _w1s * alpha1; dup[n - 2] = _w1s * alpha1; dg[n - 2] = _w1s
        elif self.top_even:
            dup[n - 1] = 0.0; dg[n - 1] = 1.0 - alpha
        else:
            dg[n - 1] = 1.0 + alpha; dup[n - 1] = 0.0
        if self.bot_sided:
            dup[0] = _w0s * alpha0; dg[0] = _w0s
            ddn[1] = _w1s * alpha1; dup[1] = _w1s * alpha1; dg[1] = _w1s
        elif self.bot_even:
            ddn[0] = 0.0; dg[0] = 1.0 - alpha
        else:
            ddn[0] = 0.0; dg[0] = 1.0 + alpha
        return _thomas(ddn, dg, dup)

    def _tri_d1_c2e(self):  # :52-98
        n, alpha = self.nE, 9.0 / 62.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        if self.top_sided:
            ddn[n - 1] = 0.0; dup[n - 1] = 0.0
            ddn[n - 2] = 1.0 / 22.0; dup[n - 2] = 1.0 / 22.0
        elif self.top_even:
            dup[n - 1] = 0.0; ddn[n - 1] = 0.0
        else:
            ddn[n - 1] = 2 * alpha; dup[n - 1] = 0.0
        if self.bot_sided:
            dup[0] = 0.0; ddn[0] = 0.0
            dup[1] = 1.0 / 22.0; ddn[1] = 1.0 / 22.0
        elif self.bot_even:
            ddn[0] = 0.0; dup[0] = 0.0
        else:
            ddn[0] = 0.0; dup[0] = 2 * alpha
        return _thomas(ddn, dg, dup)

    def _tri_d1_c2c(self):  # :100-171
        n, alpha, alpha_low = self.n, 1.0 / 3.0, 3.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        if self.top_sided:
            dup[n - 1] = _w1 * 0.0; dup[n - 2] = _w2 * _alpha_p; dup[n - 3] = _w3 * _alpha_pp
            dg[n - 1] = _w1 * 1.0; dg[n - 2] = _w2 * 1.0; dg[n - 3] = _w3 * 1.0
            ddn[n - 1] = _w1 * alpha_low; ddn[n - 2] = _w2 * _alpha_p; ddn[n - 3] = _w3 * _alpha_pp
        elif self.top_even:
            dg[n - 1] = 1.0 - alpha
        else:
            dg[n - 1] = 1.0 + alpha
        if self.bot_sided:
            ddn[0] = _w1 * 0.0; ddn[1] = _w2 * _alpha_p; ddn[2] = _w3 * _alpha_pp
            dg[0] = _w1 * 1.0; dg[1] = _w2 * 1.0; dg[2] = _w3 * 1.0
            dup[0] = _w1 * alpha_low; dup[1] = _w2 * _alpha_p; dup[2] = _w3 * _alpha_pp
        elif self.bot_even:
            dg[0] = 1.0 - alpha
        else:
            dg[0] = 1.0 + alpha
        return _thomas(ddn, dg, dup)

    def _tri_d1_e2e(self):  # :173-205
        n, alpha = self.nE, 1.0 / 3.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        dg[n - 1] = 1.0; ddn[n - 1] = 0.0 if self.top_even else 2 * alpha
        dg[0] = 1.0; dup[0] = 0.0 if self.bot_even else 2 * alpha
        return _thomas(ddn, dg, dup)

    def _tri_interp_c2e(self):  # :207-251
        n, alpha, alpha1 = self.nE, 3.0 / 10.0, 1.0 / 6.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        if self.top_sided:
            dup[n - 1] = 0.0; ddn[n - 1] = 0.0
            dup[n - 2] = alpha1; ddn[n - 2] = alpha1
        elif self.top_even:
            ddn[n - 1] = 2 * alpha; dg[n - 1] = 1.0
        else:
            ddn[n - 1] = 0.0; dg[n - 1] = 1.0
        if self.bot_sided:
            dup[0] = 0.0; ddn[0] = 0.0; dg[0] = 1.0
            dup[1] = alpha1; ddn[1] = alpha1; dg[1] = 1.0
        elif self.bot_even:
            dup[0] = 2 * alpha; dg[0] = 1.0
        else:
            dup[0] = 0.0; dg[0] = 1.0
        return _thomas(ddn, dg, dup)

    def _tri_interp_e2c(self):  # :254-296
        n, alpha, alpha0 = self.n, 3.0 / 10.0, 1.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        if self.top_sided:
            ddn[n - 1] = alpha0; dup[n - 1] = 0.0
        elif self.top_even:
            dg[n - 1] = 1.0 + alpha
        else:
            dg[n - 1] = 1.0 - alpha
        if self.bot_sided:
            dup[0] = alpha0; ddn[0] = 0.0
        elif self.bot_even:
            dg[0] = 1.0 + alpha
        else:
            dg[0] = 1.0 - alpha
        return _thomas(ddn, dg, dup)

    def _tri_d2_e2e(self):  # :299-331
        n, alpha = self.nE, 2.0 / 11.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        dg[n - 1] = 1.0; ddn[n - 1] = 2 * alpha if self.top_even else 0.0
        dg[0] = 1.0; dup[0] = 2 * alpha if self.bot_even else 0.0
        return _thomas(ddn, dg, dup)

    def _tri_d2_c2c(self):  # :333-366
        n, alpha = self.n, 2.0 / 11.0
        ddn, dg, dup = np.full(n, alpha), np.ones(n), np.full(n, alpha)
        dg[n - 1] = 1.0 + alpha if self.top_even else 1.0 - alpha
        dg[0] = 1.0 + alpha if self.bot_even else 1.0 - alpha
        return _thomas(ddn, dg, dup)

    # ---- solves ----------------------------------------------------------------------------
    @staticmethod
    def _solve_lu(y, LU, n):
        """SolveZLU_REAL (cd06stagg.F90:248-273) on rows 0..n-1 of y (planes)."""
        s1 = LU[0, 1] * y[0]
        for k in range(1, n - 1):
            y[k] = y[k] - LU[k, 0] * y[k - 1]
            s1 = s1 + LU[k, 1] * y[k]
        y[n - 1] = y[n - 1] - s1
        y[n - 1] = y[n - 1] * LU[n - 1, 2]
        y[n - 2] = y[n - 2] * LU[n - 2, 2] - y[n - 1] * LU[n - 2, 4]
        for k in range(n - 3, -1, -1):
            y[k] = y[k] * LU[k, 2] - y[k + 1] * LU[k, 3] - y[n - 1] * LU[k, 4]

    @staticmethod
    def _solve_tri(y, T):
        """SolveZTriREAL (TridiagSolver_allRoutines.F90:1-15)."""
        n = T.shape[0]
        y[0] = y[0] * T[0, 1]
        for k in range(1, n):
            y[k] = y[k] * T[k, 1] - y[k - 1] * T[k, 0]
        for k in range(n - 2, -1, -1):
            y[k] = y[k] - T[k, 2] * y[k + 1]

    # ---- right-hand sides, periodic (cd06stagg.F90:301-629) --------------------------------
    def _rhs_periodic(self, op, f):
        n = self.n
        F = lambda j: f[j - 1]  # 1-based, like the reference  # noqa: E731
        if op in ("d1_e2c", "interp_e2c"):
            if op == "d1_e2c":
                a, b = (63.0 / 62.0), (17.0 / 62.0) / 3.0
                a06, b06, sg = a * self.onebydx, b * self.onebydx, -1.0
            else:
                a, b = 3.0 / 2.0, 1.0 / 10.0
                a06, b06, sg = a * 0.5, b * 0.5, 1.0
            comb = (lambda u, v: u - v) if sg < 0 else (lambda u, v: u + v)
            r = np.empty((n,) + f.shape[1:])
            r[0] = a06 * comb(F(2), F(1)) + b06 * comb(F(3), F(n))
            r[1 : n - 1] = a06 * comb(f[2:n], f[1 : n - 1]) + b06 * comb(f[3 : n + 1], f[0 : n - 2])
            r[n - 1] = a06 * comb(F(n + 1), F(n)) + b06 * comb(F(2), F(n - 1))
            return r
        if op in ("d1_c2e", "interp_c2e"):
            if op == "d1_c2e":
                a, b = (63.0 / 62.0), (17.0 / 62.0) / 3.0
                a06, b06 = a * self.onebydx, b * self.onebydx
                comb = lambda u, v: u - v  # noqa: E731
            else:
                a, b = 3.0 / 2.0, 1.0 / 10.0
                a06, b06 = a * 0.5, b * 0.5
                comb = lambda u, v: u + v  # noqa: E731
            r = np.empty((n + 1,) + f.shape[1:])
            r[0] = a06 * comb(F(1), F(n)) + b06 * comb(F(2), F(n - 1))
            r[1] = a06 * comb(F(2), F(1)) + b06 * comb(F(3), F(n))
            r[2 : n - 1] = a06 * comb(f[2 : n - 1], f[1 : n - 2]) + b06 * comb(f[3:n], f[0 : n - 3])
            r[n - 1] = a06 * comb(F(n), F(n - 1)) + b06 * comb(F(1), F(n - 2))
            r[n] = a06 * comb(F(1), F(n)) + b06 * comb(F(2), F(n - 1))
            return r
        # second derivatives, C2C (n rows) and E2E (n + 1 rows: the last uses rows n+1, 2, 3)
        a, b = (12.0 / 11.0), (3.0 / 11.0) / 4.0
        a06, b06 = a * (self.onebydx ** 2), b * (self.onebydx ** 2)
        rows = n + 1 if op == "d2_e2e" else n
        r = np.empty((rows,) + f.shape[1:])
        r[0] = a06 * (F(2) - 2 * F(1) + F(n)) + b06 * (F(3) - 2 * F(1) + F(n - 1))
        r[1] = a06 * (F(3) - 2 * F(2) + F(1)) + b06 * (F(4) - 2 * F(2) + F(n))
        r[2 : n - 2] = (a06 * (f[3 : n - 1] - 2 * f[2 : n - 2] + f[1 : n - 3])
                        + b06 * (f[4:n] - 2 * f[2 : n - 2] + f[0 : n - 4]))
        r[n - 2] = a06 * (F(n) - 2 * F(n - 1) + F(n - 2)) + b06 * (F(1) - 2 * F(n - 1) + F(n - 3))
        r[n - 1] = a06 * (F(1) - 2 * F(n) + F(n - 1)) + b06 * (F(2) - 2 * F(n) + F(n - 2))
        if op == "d2_e2e":
            r[n] = a06 * (F(2) - 2 * F(n + 1) + F(n)) + b06 * (F(3) - 2 * F(n + 1) + F(n - 1))
        return r

    # ---- right-hand sides, non-periodic (STAGG_CD06_files/*RHS*_common.F90) -----------------
    def _rhs_nonperiodic(self, op, f):
        n, nE, dx1, dx2 = self.n, self.nE, self.onebydx, self.onebydx2
        F = lambda j: f[j - 1]  # noqa: E731
        S = lambda lo, hi: f[lo - 1 : hi]  # 1-based inclusive section  # noqa: E731
        if op == "d1_e2c":  # D1RHS_E2C_common.F90
            a, b = (63.0 / 62.0) / 1.0, (17.0 / 62.0) / 3.0
            alpha1, alpha0 = 37.0 / 183.0, -1.0
            a0, b0 = (1.0 / 24.0) * (alpha0 - 23.0), (1.0 / 8.0) * (-9.0 * alpha0 + 7.0)
            c0, d0 = (1.0 / 8.0) * (9.0 * alpha0 + 1.0), -(1.0 / 24.0) * (alpha0 + 1.0)
            a1, b1 = (3.0 / 8.0) * (3.0 - 2.0 * alpha1), (1.0 / 8.0) * (-1.0 + 22.0 * alpha1)
            a06, b06 = a * dx1, b * dx1
            r = np.empty((n,) + f.shape[1:])
            r[1 : n - 1] = b06 * (S(4, nE) - S(1, nE - 3)) + a06 * (S(3, nE - 1) - S(2, nE - 2))
            if self.bot_sided:
                r[0] = _w0s * dx1 * (a0 * F(1) + b0 * F(2) + c0 * F(3) + d0 * F(4))
                r[1] = _w1s * dx1 * ((-b1 / 3.0) * F(1) + (-a1) * F(2) + (a1) * F(3) + (b1 / 3.0) * F(4))
            elif self.bot_even:
                r[0] = b06 * (F(3) - F(2)) + a06 * (F(2) - F(1))
            else:
                r[0] = b06 * (F(3) + F(2)) + a06 * (F(2) - F(1))
            if self.top_sided:
                r[n - 1] = -_w0s * dx1 * (a0 * F(nE) + b0 * F(nE - 1) + c0 * F(nE - 2) + d0 * F(nE - 3))
                r[n - 2] = _w1s * dx1 * ((-b1 / 3.0) * F(nE - 3) + (-a1) * F(nE - 2) + (a1) * F(nE - 1)
                                         + (b1 / 3.0) * F(nE))
            elif self.top_even:
                r[n - 1] = b06 * (F(nE - 1) - F(nE - 2)) + a06 * (F(nE) - F(nE - 1))
            else:
                r[n - 1] = -b06 * (F(nE - 1) + F(nE - 2)) + a06 * (F(nE) - F(nE - 1))
            return r
        if op == "d1_c2e":  # D1RHS_C2E_common.F90
            a, b = (63.0 / 62.0) / 1.0, (17.0 / 62.0) / 3.0
            a0, b0, c0, d0 = -71.0 / 24.0, 47.0 / 8.0, -31.0 / 8.0, 23.0 / 24.0
            a1 = 12.0 / 11.0
            a06, b06 = a * dx1, b * dx1
            r = np.empty((nE,) + f.shape[1:])
            r[1 : nE - 1] = a06 * (S(2, n) - S(1, n - 1))
            r[2 : nE - 2] = r[2 : nE - 2] + b06 * (S(4, n) - S(1, n - 3))
            if self.bot_sided:
                r[0] = (a0 * F(1) + b0 * F(2) + c0 * F(3) + d0 * F(4)) * dx1
                r[1] = (F(2) - F(1)) * (a1 * dx1)
            elif self.bot_even:
                r[0] = 0.0
                r[1] = r[1] + b06 * (F(3) - F(1))
            else:
                r[0] = 2.0 * b06 * F(2) + 2.0 * a06 * F(1)
                r[1] = r[1] + b06 * (F(3) + F(1))
            if self.top_sided:
                r[nE - 2] = (F(n) - F(n - 1)) * (a1 * dx1)
                r[nE - 1] = (a0 * F(n) + b0 * F(n - 1) + c0 * F(n - 2) + d0 * F(n - 3)) * (-dx1)
            elif self.top_even:
                r[nE - 2] = r[nE - 2] + b06 * (F(n) - F(n - 2))
                r[nE - 1] = 0.0
            else:
                r[nE - 2] = r[nE - 2] - b06 * (F(n) + F(n - 2))
                r[nE - 1] = -2.0 * b06 * F(n - 1) - 2.0 * a06 * F(n)
            return r
        if op == "d1_c2c":  # D1RHS_C2C_common.F90
            a, b = (14.0 / 9.0) / 2.0, (1.0 / 9.0) / 4.0
            a06, b06 = a * dx1, b * dx1
            a_np_3, b_np_3 = _w3 * _q_pp * dx1, _w3 * _r_pp * dx1
            a_np_2 = _w2 * _q_p * dx1
            a_np_1, b_np_1 = _w1 * (-_p * dx1), _w1 * (_q * dx1)
            c_np_1, d_np_1 = _w1 * (_r * dx1), _w1 * (_s * dx1)
            r = np.empty((n,) + f.shape[1:])
            if self.bot_sided:
                r[0] = a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4)
                r[1] = a_np_2 * (F(3) - F(1))
                r[2] = a_np_3 * (F(4) - F(2)) + b_np_3 * (F(5) - F(1))
            elif self.bot_even:
                r[0] = b06 * (F(3) - F(2)) + a06 * (F(2) - F(1))
                r[1] = b06 * (F(4) - F(1)) + a06 * (F(3) - F(1))
                r[2] = b06 * (F(5) - F(1)) + a06 * (F(4) - F(2))
            else:
                r[0] = b06 * (F(3) + F(2)) + a06 * (F(2) + F(1))
                r[1] = b06 * (F(4) + F(1)) + a06 * (F(3) - F(1))
                r[2] = b06 * (F(5) - F(1)) + a06 * (F(4) - F(2))
            r[3 : n - 3] = b06 * (S(6, n - 1) - S(2, n - 5)) + a06 * (S(5, n - 2) - S(3, n - 4))
            if self.top_sided:
                r[n - 3] = a_np_3 * (F(n - 1) - F(n - 3)) + b_np_3 * (F(n) - F(n - 4))
                r[n - 2] = a_np_2 * (F(n) - F(n - 2))
                r[n - 1] = -a_np_1 * F(n) - b_np_1 * F(n - 1) - c_np_1 * F(n - 2) - d_np_1 * F(n - 3)
            elif self.top_even:
                r[n - 3] = b06 * (F(n) - F(n - 4)) + a06 * (F(n - 1) - F(n - 3))
                r[n - 2] = b06 * (F(n) - F(n - 3)) + a06 * (F(n) - F(n - 2))
                r[n - 1] = b06 * (F(n - 1) - F(n - 2)) + a06 * (F(n) - F(n - 1))
            else:
                r[n - 3] = b06 * (F(n) - F(n - 4)) + a06 * (F(n - 1) - F(n - 3))
                r[n - 2] = -b06 * (F(n) + F(n - 3)) + a06 * (F(n) - F(n - 2))
                r[n - 1] = -b06 * (F(n - 1) + F(n - 2)) - a06 * (F(n) + F(n - 1))
            return r
        if op == "d1_e2e":  # D1RHS_E2E_common.F90
            a, b = (14.0 / 9.0) / 2.0, (1.0 / 9.0) / 4.0
            a06, b06 = a * dx1, b * dx1
            r = np.empty((nE,) + f.shape[1:])
            r[1 : nE - 1] = a06 * (S(3, nE) - S(1, nE - 2))
            r[2 : nE - 2] = r[2 : nE - 2] + b06 * (S(5, nE) - S(1, nE - 4))
            if self.bot_even:
                r[0] = 0.0
                r[1] = r[1] + b06 * (F(4) - F(2))
            else:
                r[0] = b06 * (F(3) + F(3)) + a06 * (F(2) + F(2))
                r[1] = r[1] + b06 * (F(4) + F(2))
            if self.top_even:
                r[nE - 1] = 0.0
                r[nE - 2] = r[nE - 2] + b06 * (F(nE - 1) - F(nE - 3))
            else:
                r[nE - 1] = -b06 * (F(nE - 2) + F(nE - 2)) - a06 * (F(nE - 1) + F(nE - 1))
                r[nE - 2] = r[nE - 2] - b06 * (F(nE - 1) + F(nE - 3))
            return r
        if op == "d2_c2c":  # D2RHS_C2C_common.F90
            a, b = 12.0 / 11.0, (3.0 / 11.0) / 4.0
            a06, b06 = a * dx2, b * dx2
            r = np.empty((n,) + f.shape[1:])
            r[1 : n - 1] = a06 * (S(3, n) + S(1, n - 2))
            r[2 : n - 2] = r[2 : n - 2] + b06 * (S(5, n) + S(1, n - 4))
            if self.bot_even:
                r[0] = b06 * (F(3) + F(2)) + a06 * (F(2) + F(1))
                r[1] = r[1] + b06 * (F(4) + F(1))
            else:
                r[0] = b06 * (F(3) - F(2)) + a06 * (F(2) - F(1))
                r[1] = r[1] + b06 * (F(4) - F(1))
            if self.top_even:
                r[n - 1] = b06 * (F(n - 1) + F(n - 2)) + a06 * (F(n) + F(n - 1))
                r[n - 2] = r[n - 2] + b06 * (F(n) + F(n - 3))
            else:
                r[n - 1] = b06 * (-F(n - 1) + F(n - 2)) + a06 * (-F(n) + F(n - 1))
                r[n - 2] = r[n - 2] + b06 * (-F(n) + F(n - 3))
            return r - 2.0 * (b06 + a06) * f
        if op == "d2_e2e":  # D2RHS_E2E_common.F90
            a, b = 12.0 / 11.0, (3.0 / 11.0) / 4.0
            a06, b06 = a * dx2, b * dx2
            r = np.empty((nE,) + f.shape[1:])
            r[1 : nE - 1] = a06 * (S(3, nE) + S(1, nE - 2))
            r[2 : nE - 2] = r[2 : nE - 2] + b06 * (S(5, nE) + S(1, nE - 4))
            if self.bot_even:
                r[0] = b06 * (F(3) + F(3)) + a06 * (F(2) + F(2))
                r[1] = r[1] + b06 * (F(4) + F(2))
            else:
                r[0] = 0.0
                r[1] = r[1] + b06 * (F(4) - F(2))
            if self.top_even:
                r[nE - 1] = 2.0 * b06 * F(nE - 2) + 2.0 * a06 * F(nE - 1)
                r[nE - 2] = r[nE - 2] + b06 * (F(nE - 1) + F(nE - 3))
            else:
                r[nE - 1] = 0.0
                r[nE - 2] = r[nE - 2] + b06 * (-F(nE - 1) + F(nE - 3))
            return r - 2.0 * (b06 + a06) * f
        if op == "interp_c2e":  # InterpRHS_C2E_common.F90
            b, a = (1.0 / 10.0) / 2.0, (3.0 / 2.0) / 2.0
            a0, b0, c0 = 15.0 / 8.0, -5.0 / 4.0, 3.0 / 8.0
            alpha1 = 1.0 / 6.0
            a1 = (1.0 / 8.0) * (9.0 + 10.0 * alpha1)
            r = np.empty((nE,) + f.shape[1:])
            r[1 : nE - 1] = a * (S(2, n) + S(1, n - 1))
            r[2 : nE - 2] = r[2 : nE - 2] + b * (S(4, n) + S(1, n - 3))
            if self.bot_sided:
                r[0] = a0 * F(1) + b0 * F(2) + c0 * F(3)
                r[1] = (a1 / 2.0) * (F(2) + F(1))
            elif self.bot_even:
                r[0] = 2.0 * b * F(2) + 2.0 * a * F(1)
                r[1] = r[1] + b * (F(3) + F(1))
            else:
                r[0] = 0.0
                r[1] = r[1] + b * (F(3) - F(1))
            if self.top_sided:
                r[nE - 1] = a0 * F(n) + b0 * F(n - 1) + c0 * F(n - 2)
                r[nE - 2] = (a1 / 2.0) * (F(n) + F(n - 1))
            elif self.top_even:
                r[nE - 1] = 2.0 * b * F(n - 1) + 2.0 * a * F(n)
                r[nE - 2] = r[nE - 2] + b * (F(n) + F(n - 2))
            else:
                r[nE - 1] = 0.0
                r[nE - 2] = r[nE - 2] + b * (-F(n) + F(n - 2))
            return r
        # interp_e2c: InterpRHS_E2C_common.F90
        b, a = (1.0 / 10.0) / 2.0, (3.0 / 2.0) / 2.0
        alpha0 = 1.0
        a0, b0 = (1.0 / 16.0) * (5.0 - alpha0), (1.0 / 16.0) * (9.0 * alpha0 + 15.0)
        c0, d0 = (1.0 / 16.0) * (9.0 * alpha0 - 5.0), (1.0 / 16.0) * (1.0 - alpha0)
        r = np.empty((n,) + f.shape[1:])
        if self.bot_sided:
            r[0] = a0 * F(1) + b0 * F(2) + c0 * F(3) + d0 * F(4)
        elif self.bot_even:
            r[0] = b * (F(3) + F(2)) + a * (F(2) + F(1))
        else:
            r[0] = b * (F(3) - F(2)) + a * (F(2) + F(1))
        r[1 : n - 1] = b * (S(4, nE) + S(1, nE - 3)) + a * (S(3, nE - 1) + S(2, nE - 2))
        if self.top_sided:
            r[n - 1] = a0 * F(nE) + b0 * F(nE - 1) + c0 * F(nE - 2) + d0 * F(nE - 3)
        elif self.top_even:
            r[n - 1] = b * (F(nE - 1) + F(nE - 2)) + a * (F(nE) + F(nE - 1))
        else:
            r[n - 1] = b * (-F(nE - 1) + F(nE - 2)) + a * (F(nE) + F(nE - 1))
        return r

    # ---- the reference's calls (cd06stagg.F90:820-1060) -------------------------------------
    OPS = {"ddz_E2C": "d1_e2c", "ddz_C2E": "d1_c2e", "ddz_C2C": "d1_c2c", "ddz_E2E": "d1_e2e",
           "d2dz2_C2C": "d2_c2c", "d2dz2_E2E": "d2_e2e", "InterpZ_E2C": "interp_e2c", "InterpZ_C2E": "interp_c2e"}

    def apply(self, name: str, f: np.ndarray) -> np.ndarray:
        """Operator ``name`` (ddz_E2C, ..., InterpZ_C2E) on f of shape (nin, n2, n1);
        returns (nout, n2, n1).  A periodic object has no C2C / E2E first
        derivative (the reference solves those with the non-periodic tables,
        which a periodic init never allocates)."""
        op = self.OPS[name]
        n, nE = self.n, self.nE
        f = np.asarray(f, dtype=np.float64)
        if self.periodic:
            if op in ("d1_c2c", "d1_e2e"):
                raise ValueError(f"{name} needs a non-periodic cd06stagg")
            y = self._rhs_periodic(op, f)
            LU = {"d1": self.LU_D1, "d2": self.LU_D2, "in": self.LU_interp}[op[:2]]
            self._solve_lu(y, LU, n)
            if y.shape[0] == nE:
                y[nE - 1] = y[0]
            return y
        y = self._rhs_nonperiodic(op, f)
        self._solve_tri(y, self.tri[op])
        return y
