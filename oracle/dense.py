"""Dense assembly of the reference operators (TEST INFRASTRUCTURE ONLY).

An independent second transcription of the reference's band definitions and
right-hand-side stencils, as explicit n x n matrices:

    D = A^{-1} B        (one axis; D_x = I (x) I (x) D by Kronecker structure)

* A: the left-hand side the reference factorises -- cd06.F90:148-195 and
  :264-327 (cyclic tridiagonal alpha/1/alpha, or the bounded Tri1 bands),
  cd10.F90:214-310, :429-556, :580-686 (cyclic pentadiagonal beta/alpha/1/
  alpha/beta, or the bounded penta1/penta2 bands), cf90.F90:118-170, :276-396.
* B: the explicit stencils ComputeXD1RHS / ComputeXD2RHS / ComputeXRHS
  (cd06.F90:515-592, cd10.F90:1098-1263 and 1587-1736, cf90.F90:610-804),
  row by row.

Used by the tests to cross-check the C restatement's LU/Thomas sweeps and to
form D^T for the adjoint checks.  Nothing here factorises like the reference:
it is plain numpy linear algebra.
"""
from __future__ import annotations

import numpy as np

CD06, CD10, CF90 = 0, 1, 2
FILTER, D1, D2 = 0, 1, 2

# cd06.F90:14-59
A06, B06, AL06 = (14.0 / 9.0) / 2.0, (1.0 / 9.0) / 4.0, 1.0 / 3.0
_c6 = dict(alpha=3.0, p=17.0 / 6.0, q=1.5, r=1.5, s=-1.0 / 6.0, ah=1.0 / 3.0, qp=0.75, ap=0.25)
_c6["app"] = (((40 * _c6["ah"] - 1) * _c6["q"] + 7 * (4 * _c6["ah"] - 1) * _c6["s"])
              / (16 * (_c6["ah"] + 2) * _c6["q"] + 8 * (1 - 4 * _c6["ah"]) * _c6["s"]))
_c6["qpp"] = (1.0 / 3.0) * (_c6["app"] + 2)
_c6["rpp"] = (1.0 / 12.0) * (4 * _c6["app"] - 1)
_c6["w1"] = (2 * _c6["ah"] + 1) / (2 * (_c6["q"] + _c6["s"]))
_c6["w2"] = (((8 * _c6["ah"] + 7) * _c6["q"] - 6 * (2 * _c6["ah"] + 1) * _c6["r"] + (8 * _c6["ah"] + 7) * _c6["s"])
             / (9 * (_c6["q"] + _c6["s"])))
_c6["w3"] = (4 * (_c6["ah"] + 2) * _c6["q"] + 2 * (1 - 4 * _c6["ah"]) * _c6["s"]) / (9 * (_c6["q"] + _c6["s"]))

# cd10.F90:16-104
AL1, BE1 = 0.5, 1.0 / 20.0
A1, B1, C1 = (17.0 / 12.0) / 2.0, (101.0 / 150.0) / 4.0, (1.0 / 100.0) / 6.0
AL2, BE2 = 334.0 / 899.0, 43.0 / 1798.0
A2, B2, C2 = 1065.0 / 1798.0, (1038.0 / 899.0) / 4.0, (79.0 / 1798.0) / 9.0
_k = dict(alpha=3.0, p=-17.0 / 6.0, q=1.5, r=1.5, s=-1.0 / 6.0, qh=A1, rh=B1, sh=C1, ah=AL1, bh=BE1, qp=0.75, ap=0.25)
_k["appp"] = (8 * _k["rh"] - 175 * _k["sh"]) / (18 * _k["rh"] - 550 * _k["sh"])
_k["bppp"] = (1.0 / 20.0) * (-3 + 8 * _k["appp"])
_k["qppp"] = (1.0 / 12.0) * (12 - 7 * _k["appp"])
_k["rppp"] = (1.0 / 600.0) * (568 * _k["appp"] - 183)
_k["sppp"] = (1.0 / 300.0) * (9 * _k["appp"] - 4)
_t1 = _k["s"] * (_k["rh"] + 2 * _k["sh"]) - _k["q"] * (_k["qh"] + _k["rh"] + _k["sh"])
_t2 = _k["qh"] + _k["rh"] - _k["sh"] * (_k["qppp"] / _k["sppp"] - 1)
_k["app"] = (((17 * _t1) / (72 * (_k["q"] + _k["s"]) * _t2) - 8.0 / 9.0)
             / ((19 * _t1) / (24 * (_k["q"] + _k["s"]) * _t2) - 1.0 / 3))
_k["bpp"] = (1.0 / 12.0) * (-1 + 3 * _k["app"])
_k["qpp"] = (2.0 / 18.0) * (8 - 3 * _k["app"])
_k["rpp"] = (1.0 / 72.0) * (-17 + 57 * _k["app"])
_k["w1"] = (_k["qh"] + 2 * _k["rh"] + 3 * _k["sh"]) / (_k["q"] + _k["s"])
_k["w2"] = (1 / _k["qp"]) * (_k["rh"] + _k["sh"] * (1 + _k["qppp"] / _k["sppp"])
                              - _k["r"] * (_k["qh"] + 2 * _k["rh"] + 3 * _k["sh"]) / (_k["q"] + _k["s"]))
_k["w3"] = (_k["qh"] + _k["rh"] + _k["sh"] * (1 - _k["qppp"] / _k["sppp"])) / _k["rpp"]
_k["w4"] = _k["sh"] / _k["sppp"]
_b1a = 11.0
_d2b = dict(a1=(11 * _b1a + 35) / 12, b1=-(5 * _b1a + 26) / 3, c1=(_b1a + 19) / 2, d1=(_b1a - 14) / 3,
            e1=(11 - _b1a) / 12, al1=_b1a, al2=0.1, a2=(4 * (1 - 0.1) / 3),
            al3=344.0 / 1179.0)
_d2b["be3"] = (38.0 * _d2b["al3"] - 9.0) / 214.0
_d2b["a3"] = (696 - 1191 * _d2b["al3"]) / 428
_d2b["b3"] = ((2454 * _d2b["al3"] - 294) / 535) / 4.0

# cf90.F90:16-48
AL9, BE9 = 0.66624, 0.16688
CF = (0.99965, 0.66652, 0.16674, 4.0e-5, -5.0e-6)
CF2 = dict(al=0.4997, a=0.9997, b=0.49985)
CF3 = dict(al=0.66624, be=0.16688, a=0.99952, b=0.66656, c=0.1668)
CF4 = dict(al=0.66624, be=0.16688, a=0.99968, b=0.66652, c=0.16672, d=4.0e-5)


def _cyclic(n: int, diag: list[float]) -> np.ndarray:
    """Circulant band matrix; diag = coefficients for offsets -m..m."""
    m = len(diag) // 2
    A = np.zeros((n, n))
    for i in range(n):
        for o, c in zip(range(-m, m + 1), diag):
            A[i, (i + o) % n] += c
    return A


def _banded(n: int, bands: dict[int, np.ndarray]) -> np.ndarray:
    A = np.zeros((n, n))
    for o, v in bands.items():
        for i in range(n):
            j = i + o
            if 0 <= j < n:
                A[i, j] = v[i]
    return A


def lhs(scheme: int, kind: int, n: int, periodic: bool, bc1: int = 0, bcn: int = 0) -> np.ndarray:
    """The left-hand-side matrix A."""
    if scheme == CD06:
        if periodic:
            return _cyclic(n, [AL06, 1.0, AL06])
        a = np.full(n, AL06); b = np.ones(n); c = np.full(n, AL06)
        w1, w2, w3, ap, app, al = _c6["w1"], _c6["w2"], _c6["w3"], _c6["ap"], _c6["app"], _c6["alpha"]
        if bc1 == 0:
            a[0:3] = [0.0, w2 * ap, w3 * app]; b[0:3] = [w1, w2, w3]; c[0:3] = [w1 * al, w2 * ap, w3 * app]
        if bcn == 0:
            c[n - 3:] = [w3 * app, w2 * ap, 0.0]; b[n - 3:] = [w3, w2, w1]; a[n - 3:] = [w3 * app, w2 * ap, w1 * al]
        return _banded(n, {-1: a, 0: b, 1: c})
    if scheme == CD10:
        al, be = (AL1, BE1) if kind == D1 else (AL2, BE2)
    else:
        al, be = AL9, BE9
    if periodic:
        return _cyclic(n, [be, al, 1.0, al, be])
    bt = np.full(n, be); b = np.full(n, al); d = np.ones(n); a = np.full(n, al); at = np.full(n, be)

    def row(i, vals):
        bt[i], b[i], d[i], a[i], at[i] = vals

    if scheme == CD10 and kind == D1:
        k = _k
        closure = [(k["w1"], (0, 0, 1, k["alpha"], 0)), (k["w2"], (0, k["ap"], 1, k["ap"], 0)),
                   (k["w3"], (k["bpp"], k["app"], 1, k["app"], k["bpp"])),
                   (k["w4"], (k["bppp"], k["appp"], 1, k["appp"], k["bppp"]))]
        if bc1 == 0:
            for r, (w, v) in enumerate(closure):
                row(r, [w * x for x in v])
        elif bc1 == 1:
            row(0, (0, 0, 1, 0, 0)); row(1, (0, al, 1 - be, al, be))
        else:
            row(0, (0, 0, 1, 2 * al, 2 * be)); row(1, (0, al, 1 + be, al, be))
        if bcn == 0:
            for r, (w, v) in enumerate(closure):
                row(n - 1 - r, [w * x for x in v[::-1]])
        elif bcn == 1:
            row(n - 1, (0, 0, 1, 0, 0)); row(n - 2, (be, al, 1 - be, al, 0))
        else:
            row(n - 1, (2 * be, 2 * al, 1, 0, 0)); row(n - 2, (be, al, 1 + be, al, 0))
    elif scheme == CD10:
        q = _d2b
        if bc1 == 0:
            row(0, (0, 0, 1, q["al1"], 0)); row(1, (0, q["al2"], 1, q["al2"], 0))
            row(2, (q["be3"], q["al3"], 1, q["al3"], q["be3"]))
        elif bc1 == 1:
            row(0, (0, 0, 1, 2 * al, 2 * be)); row(1, (0, al, 1 + be, al, be))
        else:
            row(0, (0, 0, 1, 0, 0)); row(1, (0, al, 1 - be, al, be))
        if bcn == 0:
            row(n - 3, (q["be3"], q["al3"], 1, q["al3"], q["be3"])); row(n - 2, (0, q["al2"], 1, q["al2"], 0))
            row(n - 1, (0, q["al1"], 1, 0, 0))
        elif bcn == 1:
            row(n - 2, (be, al, 1 + be, al, 0)); row(n - 1, (2 * be, 2 * al, 1, 0, 0))
        else:
            row(n - 2, (be, al, 1 - be, al, 0)); row(n - 1, (0, 0, 1, 0, 0))
    else:
        if bc1 == 0:
            row(0, (0, 0, 1, 0, 0)); row(1, (0, CF2["al"], 1, CF2["al"], 0))
            row(2, (CF3["be"], CF3["al"], 1, CF3["al"], CF3["be"])); row(3, (CF4["be"], CF4["al"], 1, CF4["al"], CF4["be"]))
        elif bc1 == 1:
            row(0, (0, 0, 1, 2 * al, 2 * be)); row(1, (0, al, 1 + be, al, be))
        else:
            row(0, (0, 0, 1, 0, 0)); row(1, (0, al, 1 - be, al, be))
        if bcn == 0:
            row(n - 1, (0, 0, 1, 0, 0)); row(n - 2, (0, CF2["al"], 1, CF2["al"], 0))
            row(n - 3, (CF3["be"], CF3["al"], 1, CF3["al"], CF3["be"])); row(n - 4, (CF4["be"], CF4["al"], 1, CF4["al"], CF4["be"]))
        elif bcn == 1:
            row(n - 1, (2 * be, 2 * al, 1, 0, 0)); row(n - 2, (be, al, 1 + be, al, 0))
        else:
            row(n - 1, (0, 0, 1, 0, 0)); row(n - 2, (be, al, 1 - be, al, 0))
    return _banded(n, {-2: bt, -1: b, 0: d, 1: a, 2: at})


class _Rows:
    """Accumulates B row by row from (coefficient, [(column, sign), ...]) terms, 1-based."""

    def __init__(self, n: int):
        self.n = n
        self.B = np.zeros((n, n))

    def add(self, i: int, *terms):
        for c, cols in terms:
            for j, sgn in cols:
                self.B[i - 1, (j - 1) % self.n] += sgn * c


def _anti(c, i, d):
    return (c, [(i + d, 1), (i - d, -1)])


def _sym2(c, i, d):
    return (c, [(i + d, 1), (i, -2), (i - d, 1)])


def _sym(c, i, d):
    return (c, [(i + d, 1), (i - d, 1)])


def rhs(scheme: int, kind: int, n: int, dx: float, periodic: bool, bc1: int = 0, bcn: int = 0) -> np.ndarray:
    """The right-hand-side stencil matrix B."""
    R = _Rows(n)
    ob, ob2 = 1.0 / dx, (1.0 / dx) / dx
    if scheme == CD06:
        a06, b06 = A06 * ob, B06 * ob
        if periodic:
            for i in range(1, n + 1):
                R.add(i, _anti(a06, i, 1), _anti(b06, i, 2))
            return R.B
        c = _c6
        a3, b3, a2 = c["w3"] * c["qpp"] * ob, c["w3"] * c["rpp"] * ob, c["w2"] * c["qp"] * ob
        n1 = [c["w1"] * (-c["p"] * ob), c["w1"] * (c["q"] * ob), c["w1"] * (c["r"] * ob), c["w1"] * (c["s"] * ob)]
        R.add(1, *[(n1[m], [(1 + m, 1)]) for m in range(4)])
        R.add(2, _anti(a2, 2, 1)); R.add(3, _anti(a3, 3, 1), _anti(b3, 3, 2))
        for i in range(4, n - 2):
            R.add(i, _anti(b06, i, 2), _anti(a06, i, 1))
        R.add(n - 2, _anti(a3, n - 2, 1), _anti(b3, n - 2, 2)); R.add(n - 1, _anti(a2, n - 1, 1))
        R.add(n, *[(n1[m], [(n - m, -1)]) for m in range(4)])
        return R.B
    if scheme == CD10 and kind == D1:
        a, b, c = A1 * ob, B1 * ob, C1 * ob
        if periodic:
            for i in range(1, n + 1):
                R.add(i, _anti(a, i, 1), _anti(b, i, 2), _anti(c, i, 3))
            return R.B
        k = _k
        a4, b4, c4 = k["w4"] * k["qppp"] * ob, k["w4"] * k["rppp"] * ob, k["w4"] * k["sppp"] * ob
        a3, b3, a2 = k["w3"] * k["qpp"] * ob, k["w3"] * k["rpp"] * ob, k["w2"] * k["qp"] * ob
        n1 = [k["w1"] * (k["p"] * ob), k["w1"] * (k["q"] * ob), k["w1"] * (k["r"] * ob), k["w1"] * (k["s"] * ob)]
        if bc1 == 0:
            R.add(1, *[(n1[m], [(1 + m, 1)]) for m in range(4)])
            R.add(2, _anti(a2, 2, 1)); R.add(3, _anti(a3, 3, 1), _anti(b3, 3, 2))
            R.add(4, _anti(a4, 4, 1), _anti(b4, 4, 2), _anti(c4, 4, 3))
        elif bc1 == 1:
            R.add(2, (a, [(3, 1), (1, -1)]), (b, [(4, 1), (2, -1)]), (c, [(5, 1), (3, -1)]))
            R.add(3, (a, [(4, 1), (2, -1)]), (b, [(5, 1), (1, -1)]), (c, [(6, 1), (2, -1)]))
            R.add(4, _anti(a, 4, 1), _anti(b, 4, 2), _anti(c, 4, 3))
        else:
            R.add(1, (a, [(2, 1), (2, 1)]), (b, [(3, 1), (3, 1)]), (c, [(4, 1), (4, 1)]))
            R.add(2, (a, [(3, 1), (1, -1)]), (b, [(4, 1), (2, 1)]), (c, [(5, 1), (3, 1)]))
            R.add(3, (a, [(4, 1), (2, -1)]), (b, [(5, 1), (1, -1)]), (c, [(6, 1), (2, 1)]))
            R.add(4, _anti(a, 4, 1), _anti(b, 4, 2), _anti(c, 4, 3))
        for i in range(5, n - 3):
            R.add(i, _anti(a, i, 1), _anti(b, i, 2), _anti(c, i, 3))
        if bcn == 0:
            R.add(n - 3, _anti(a4, n - 3, 1), _anti(b4, n - 3, 2), _anti(c4, n - 3, 3))
            R.add(n - 2, _anti(a3, n - 2, 1), _anti(b3, n - 2, 2)); R.add(n - 1, _anti(a2, n - 1, 1))
            R.add(n, *[(n1[m], [(n - m, -1)]) for m in range(4)])
        elif bcn == 1:
            R.add(n - 3, _anti(a, n - 3, 1), _anti(b, n - 3, 2), _anti(c, n - 3, 3))
            R.add(n - 2, (a, [(n - 1, 1), (n - 3, -1)]), (b, [(n, 1), (n - 4, -1)]), (c, [(n - 1, 1), (n - 5, -1)]))
            R.add(n - 1, (a, [(n, 1), (n - 2, -1)]), (b, [(n - 1, 1), (n - 3, -1)]), (c, [(n - 2, 1), (n - 4, -1)]))
        else:
            R.add(n - 3, _anti(a, n - 3, 1), _anti(b, n - 3, 2), _anti(c, n - 3, 3))
            R.add(n - 2, (a, [(n - 1, 1), (n - 3, -1)]), (b, [(n, 1), (n - 4, -1)]), (c, [(n - 1, -1), (n - 5, -1)]))
            R.add(n - 1, (a, [(n, 1), (n - 2, -1)]), (b, [(n - 1, -1), (n - 3, -1)]), (c, [(n - 2, -1), (n - 4, -1)]))
            R.add(n, (a, [(n - 1, -1), (n - 1, -1)]), (b, [(n - 2, -1), (n - 2, -1)]), (c, [(n - 3, -1), (n - 3, -1)]))
        return R.B
    if scheme == CD10:
        a, b, c = A2 * ob2, B2 * ob2, C2 * ob2
        if periodic:
            for i in range(1, n + 1):
                R.add(i, _sym2(a, i, 1), _sym2(b, i, 2), _sym2(c, i, 3))
            return R.B
        q = _d2b
        a3, b3, a2 = q["a3"] * ob2, q["b3"] * ob2, q["a2"] * ob2
        e1 = [q["a1"] * ob2, q["b1"] * ob2, q["c1"] * ob2, q["d1"] * ob2, q["e1"] * ob2]
        if bc1 == 0:
            R.add(1, *[(e1[m], [(1 + m, 1)]) for m in range(5)])
            R.add(2, _sym2(a2, 2, 1)); R.add(3, _sym2(a3, 3, 1), _sym2(b3, 3, 2))
        elif bc1 == 1:
            R.add(1, (a, [(2, 1), (1, -2), (2, 1)]), (b, [(3, 1), (1, -2), (3, 1)]), (c, [(4, 1), (1, -2), (4, 1)]))
            R.add(2, (a, [(3, 1), (2, -2), (1, 1)]), (b, [(4, 1), (2, -2), (2, 1)]), (c, [(5, 1), (2, -2), (3, 1)]))
            R.add(3, (a, [(4, 1), (3, -2), (2, 1)]), (b, [(5, 1), (3, -2), (1, 1)]), (c, [(6, 1), (3, -2), (2, 1)]))
        else:
            R.add(1, (a, [(2, 1), (1, -2), (2, -1)]), (b, [(3, 1), (1, -2), (3, -1)]), (c, [(4, 1), (1, -2), (4, -1)]))
            R.add(2, (a, [(3, 1), (2, -2), (1, 1)]), (b, [(4, 1), (2, -2), (2, -1)]), (c, [(5, 1), (2, -2), (3, -1)]))
            R.add(3, (a, [(4, 1), (3, -2), (2, 1)]), (b, [(5, 1), (3, -2), (1, 1)]), (c, [(6, 1), (3, -2), (2, -1)]))
        for i in range(4, n - 2):
            R.add(i, _sym2(a, i, 1), _sym2(b, i, 2), _sym2(c, i, 3))
        if bcn == 0:
            R.add(n - 2, _sym2(a3, n - 2, 1), _sym2(b3, n - 2, 2)); R.add(n - 1, _sym2(a2, n - 1, 1))
            R.add(n, *[(e1[m], [(n - m, 1)]) for m in range(5)])
        elif bcn == 1:
            R.add(n - 2, (a, [(n - 1, 1), (n - 2, -2), (n - 3, 1)]), (b, [(n, 1), (n - 2, -2), (n - 4, 1)]),
                  (c, [(n - 1, 1), (n - 2, -2), (n - 5, 1)]))
            R.add(n - 1, (a, [(n, 1), (n - 1, -2), (n - 2, 1)]), (b, [(n - 1, 1), (n - 1, -2), (n - 3, 1)]),
                  (c, [(n - 2, 1), (n - 1, -2), (n - 4, 1)]))
            R.add(n, (a, [(n - 1, 1), (n, -2), (n - 1, 1)]), (b, [(n - 2, 1), (n, -2), (n - 2, 1)]),
                  (c, [(n - 3, 1), (n, -2), (n - 3, 1)]))
        else:
            R.add(n - 2, (a, [(n - 1, 1), (n - 2, -2), (n - 3, 1)]), (b, [(n, 1), (n - 2, -2), (n - 4, 1)]),
                  (c, [(n - 1, -1), (n - 2, -2), (n - 5, 1)]))
            R.add(n - 1, (a, [(n, 1), (n - 1, -2), (n - 2, 1)]), (b, [(n - 1, -1), (n - 1, -2), (n - 3, 1)]),
                  (c, [(n - 2, -1), (n - 1, -2), (n - 4, 1)]))
            R.add(n, (a, [(n - 1, -1), (n, -2), (n - 1, 1)]), (b, [(n - 2, -1), (n, -2), (n - 2, 1)]),
                  (c, [(n - 3, -1), (n, -2), (n - 3, 1)]))
        return R.B
    # cf90
    a9, b9, c9, d9, e9 = CF
    coef = [b9, c9, d9, e9]
    if periodic:
        for i in range(1, n + 1):
            R.add(i, (a9, [(i, 1)]), *[_sym(coef[m], i, m + 1) for m in range(4)])
        return R.B
    if bc1 == 0:
        R.add(1, (1.0, [(1, 1)]))
        R.add(2, (CF2["a"], [(2, 1)]), _sym(CF2["b"], 2, 1))
        R.add(3, (CF3["a"], [(3, 1)]), _sym(CF3["b"], 3, 1), _sym(CF3["c"], 3, 2))
        R.add(4, (CF4["a"], [(4, 1)]), _sym(CF4["b"], 4, 1), _sym(CF4["c"], 4, 2), _sym(CF4["d"], 4, 3))
    else:
        sg = 1 if bc1 == 1 else -1
        # mirror about node 1: f(1-m) -> sg * f(1+m)
        for i in range(1, 5):
            terms = [(a9, [(i, 1)])]
            for m in range(1, 5):
                lo = i - m
                cols = [(i + m, 1), (lo, 1) if lo >= 1 else (2 - lo, sg)]
                terms.append((coef[m - 1], cols))
            R.add(i, *terms)
    for i in range(5, n - 3):
        R.add(i, (a9, [(i, 1)]), *[_sym(coef[m], i, m + 1) for m in range(4)])
    if bcn == 0:
        R.add(n - 3, (CF4["a"], [(n - 3, 1)]), _sym(CF4["b"], n - 3, 1), _sym(CF4["c"], n - 3, 2), _sym(CF4["d"], n - 3, 3))
        R.add(n - 2, (CF3["a"], [(n - 2, 1)]), _sym(CF3["b"], n - 2, 1), _sym(CF3["c"], n - 2, 2))
        R.add(n - 1, (CF2["a"], [(n - 1, 1)]), _sym(CF2["b"], n - 1, 1))
        R.add(n, (1.0, [(n, 1)]))
    else:
        sg = 1 if bcn == 1 else -1
        # mirror about node n: f(n+m) -> sg * f(n-m)
        for i in range(n - 3, n + 1):
            terms = [(a9, [(i, 1)])]
            for m in range(1, 5):
                hi = i + m
                cols = [(hi, 1) if hi <= n else (2 * n - hi, sg), (i - m, 1)]
                terms.append((coef[m - 1], cols))
            R.add(i, *terms)
    return R.B


def operator(scheme: int, kind: int, n: int, dx: float, periodic: bool, bc1: int = 0, bcn: int = 0) -> np.ndarray:
    """D = A^{-1} B for one axis (dense, n x n)."""
    if n == 1:
        return np.eye(1) if kind == FILTER else np.zeros((1, 1))
    A = lhs(scheme, kind, n, periodic, bc1, bcn)
    B = rhs(scheme, kind, n, dx, periodic, bc1, bcn)
    return np.linalg.solve(A, B)


def apply_axis(D: np.ndarray, f: np.ndarray, axis: int) -> np.ndarray:
    """Apply the 1-D operator D along `axis` (1=x, 2=y, 3=z) of a field stored
    as a C-ordered (n3, n2, n1) array (column-major (n1, n2, n3))."""
    ax = {1: 2, 2: 1, 3: 0}[axis]
    return np.moveaxis(np.tensordot(D, np.moveaxis(f, ax, 0), axes=(1, 0)), 0, ax)
