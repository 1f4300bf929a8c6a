"""Closed forms and test recipes of the reference, restated for the parity tests.

* ``mod_wavenumber``: the modified wavenumbers / transfer function of
  src/utilities/spectral.F90:938-1010 (GetCF90TransferFunction,
  GetCD10ModWaveNum, GetCD10D2ModWaveNum, GetCD06ModWaveNum).
* ``reference_recipes``: the reference tests tests/test_cd06.F90,
  test_cd10.F90, test_cd10_NP.F90, test_cd10_der2.F90, test_cf90.F90,
  test_filters.F90 and test_filters_NP.F90 as written -- the same sizes,
  grids, functions, closures and comparisons.  Each check carries the
  quantity the reference test prints and, where one exists, the discrete
  operator's exact output in closed form.
* ``closure_pins``: closed-form known answers for every bounded closure pair
  (bc1, bcn) in {0, 1, -1}^2 of cd10 d1, cd10 d2 and cf90 (and cd06's (0, 0)):
  a closure of formal order p reproduces polynomials of degree <= p exactly,
  and a symmetric (bc = 1) or antisymmetric (bc = -1) closure reproduces a
  Fourier mode with that parity about the boundary node exactly, because the
  mirrored extension is then the mode itself.

Every check is a ``Check``; ``apply`` callbacks compute the operator on it, so
the same recipes run through the oracle on the CPU and through the CUDA path.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass
from typing import Callable, Iterator, Optional

import numpy as np

import oracle

CD06, CD10, CF90 = oracle.CD06, oracle.CD10, oracle.CF90
FILTER, D1, D2 = oracle.FILTER, oracle.D1, oracle.D2


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
    if scheme == CD06:  # spectral.F90:987-1010
        alpha = 1.0 / 3.0
        a, b = (2.0 / 9.0) * (8 - 3 * alpha), (1.0 / 18.0) * (-17 + 57 * alpha)
        return (a * np.sin(w) + (b / 2) * np.sin(2 * w)) / (1 + 2 * alpha * np.cos(w)) / dx
    d1, d2 = _cd10_consts()
    if scheme == CD10 and kind == D1:  # spectral.F90:950-961
        c = d1
        num = 2 * c["a"] * np.sin(w) + 2 * c["b"] * np.sin(2 * w) + 2 * c["c"] * np.sin(3 * w)
        return num / (1 + 2 * c["alpha"] * np.cos(w) + 2 * c["beta"] * np.cos(2 * w)) / dx
    if scheme == CD10:  # spectral.F90:965-984 (which returns this times dx)
        c = d2
        a, b, cc = c["a"], c["b"] * 4, c["c"] * 9
        num = 2 * a * (1 - np.cos(w)) + (b / 2) * (1 - np.cos(2 * w)) + (2 * cc / 9) * (1 - np.cos(3 * w))
        return num / (1 + 2 * c["alpha"] * np.cos(w) + 2 * c["beta"] * np.cos(2 * w)) / dx ** 2
    # cf90 transfer function, spectral.F90:938-948 and the reference tests'
    # GetTransferFunction (tests/test_cf90.F90:106-115), cf90.F90:16-22 constants
    alpha, beta = 6.6624e-1, 1.6688e-1
    a, b, c, d, e = 9.9965e-1, 6.6652e-1, 1.6674e-1, 4.0e-5, -5.0e-6
    num = a + 2 * b * np.cos(w) + 2 * c * np.cos(2 * w) + 2 * d * np.cos(3 * w) + 2 * e * np.cos(4 * w)
    return num / (1 + 2 * alpha * np.cos(w) + 2 * beta * np.cos(2 * w))


@dataclass
class Check:
    """One operator application of a recipe.

    ``f`` is the field as a C-ordered (n3, n2, n1) array (the reference's
    f(n1, n2, n3)); the operator acts along ``axis`` with ``n`` points and
    spacing ``dx`` (1 for the filter); ``bc`` is the (bc1, bcn) the call
    passes (and the init closures, for cd06).  ``exact`` is what the
    reference test compares against, ``closed`` the discrete operator's exact
    output when it is known in closed form (else None); ``signed`` marks a
    test that prints MAXVAL(df - exact) rather than MAXVAL(ABS(df - exact)).
    """

    name: str
    source: str
    scheme: int
    kind: int
    axis: int
    n: int
    dx: float
    periodic: bool
    bc: tuple
    f: np.ndarray
    exact: np.ndarray
    closed: Optional[np.ndarray]
    signed: bool = False

    @property
    def na_nb(self) -> tuple:
        n3, n2, n1 = self.f.shape
        return {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[self.axis]

    def printed(self, got: np.ndarray) -> float:
        """The error the reference test prints for output ``got``."""
        d = got - self.exact
        return float(d.max() if self.signed else np.abs(d).max())

    def closed_err(self, got: np.ndarray) -> float:
        """max |got - closed| / max |closed| (the filter's against max |f| too;
        an identically zero answer is compared absolutely)."""
        scale = float(np.abs(self.closed).max())
        if self.kind == FILTER:
            scale = max(scale, float(np.abs(self.f).max()))
        return float(np.abs(got - self.closed).max()) / (scale if scale > 0 else 1.0)


def oracle_apply(c: Check) -> np.ndarray:
    """The oracle's output for a check, shaped like ``c.f``."""
    ib = c.bc if c.scheme == CD06 else (0, 0)
    o = oracle.OracleOp(c.scheme, c.n, c.dx, c.periodic, *ib)
    na, nb = c.na_nb
    return o.apply(c.kind, c.axis, c.f, na, nb, *c.bc).reshape(c.f.shape)


def _axes(nx, ny, nz, dx, dy, dz):
    x = (np.arange(nx) * dx)[None, None, :]
    y = (np.arange(ny) * dy)[None, :, None]
    z = (np.arange(nz) * dz)[:, None, None]
    return x, y, z


def _full(a, shape):
    out = np.empty(shape)
    out[...] = a
    return out


def reference_recipes(large: bool = True) -> Iterator[Check]:
    """The reference tests' recipes as written, one Check per printed error.

    ``large=False`` skips the three 256^3 recipes (test_cd06, test_filters,
    test_filters_NP)."""
    two_pi = 2 * np.pi
    # tests/test_cd06.F90:9-50: periodic 256^3, dx = 2 pi/256, f = sin(x);
    # dd1 against cos(x), dd2 and dd3 against 0 (f does not vary along y, z)
    if large:
        n = 256
        dx = two_pi / n
        x, y, z = _axes(n, n, n, dx, dx, dx)
        sh = (n, n, n)
        f = _full(np.sin(x), sh)
        kp = mod_wavenumber(CD06, D1, 1, dx)
        yield Check("test_cd06:dd1", "tests/test_cd06.F90:38-40", CD06, D1, 1, n, dx, True, (0, 0), f,
                    _full(np.cos(x), sh), _full(kp * np.cos(x), sh))
        zero = np.zeros(sh)
        yield Check("test_cd06:dd2", "tests/test_cd06.F90:44-46", CD06, D1, 2, n, dx, True, (0, 0), f, zero, zero)
        yield Check("test_cd06:dd3", "tests/test_cd06.F90:50-52", CD06, D1, 3, n, dx, True, (0, 0), f, zero, zero)
        del f, zero
    # tests/test_cd10.F90:9-80: periodic 32^3, dx = 2 pi/32,
    # f = sin x + sin y + sin z; first and second derivative along each axis
    n = 32
    dx = two_pi / n
    x, y, z = _axes(n, n, n, dx, dx, dx)
    sh = (n, n, n)
    f = _full(np.sin(x) + np.sin(y) + np.sin(z), sh)
    k1, k2 = mod_wavenumber(CD10, D1, 1, dx), mod_wavenumber(CD10, D2, 1, dx)
    lines = {1: "57-63", 2: "66-72", 3: "75-81"}
    for axis, c in ((1, x), (2, y), (3, z)):
        src = f"tests/test_cd10.F90:{lines[axis]}"
        yield Check(f"test_cd10:dd{axis}", src, CD10, D1, axis, n, dx, True, (0, 0), f,
                    _full(np.cos(c), sh), _full(k1 * np.cos(c), sh))
        yield Check(f"test_cd10:d2d{axis}", src, CD10, D2, axis, n, dx, True, (0, 0), f,
                    _full(-np.sin(c), sh), _full(-k2 * np.sin(c), sh))
    # tests/test_cd10_NP.F90:9-83: bounded 32^3, dx = (pi/2)/31, f = cos x cos y cos z,
    # closures (1, -1): f is even about 0 and odd about pi/2, which the symmetric and
    # antisymmetric closures reproduce exactly
    n = 32
    dx = (np.pi / 2) / (n - 1)
    x, y, z = _axes(n, n, n, dx, dx, dx)
    cx, cy, cz = np.cos(x), np.cos(y), np.cos(z)
    f = _full(cx * cy * cz, sh)
    k1, k2 = mod_wavenumber(CD10, D1, 1, dx), mod_wavenumber(CD10, D2, 1, dx)
    lines = {1: "57-63", 2: "66-72", 3: "75-81"}
    for axis, c in ((1, x), (2, y), (3, z)):
        others = {1: cy * cz, 2: cx * cz, 3: cx * cy}[axis]
        src = f"tests/test_cd10_NP.F90:{lines[axis]}"
        yield Check(f"test_cd10_NP:dd{axis}", src, CD10, D1, axis, n, dx, False, (1, -1), f,
                    _full(-np.sin(c) * others, sh), _full(-k1 * np.sin(c) * others, sh))
        yield Check(f"test_cd10_NP:d2d{axis}", src, CD10, D2, axis, n, dx, False, (1, -1), f,
                    _full(-np.cos(c) * others, sh), _full(-k2 * np.cos(c) * others, sh))
    # tests/test_cd10_der2.F90:1-34: bounded init(32, 2 pi/32, .false., 0, 0) on a
    # 32 x 1 x 1 field, f = cos x; d2d1 against -cos x, dd1 against -sin x
    n = 32
    dx = two_pi / n
    x = np.arange(n) * dx
    f = np.cos(x).reshape(1, 1, n)
    yield Check("test_cd10_der2:d2d1", "tests/test_cd10_der2.F90:20-28", CD10, D2, 1, n, dx, False, (0, 0), f,
                -np.cos(x).reshape(1, 1, n), None)
    yield Check("test_cd10_der2:dd1", "tests/test_cd10_der2.F90:29-32", CD10, D1, 1, n, dx, False, (0, 0), f,
                -np.sin(x).reshape(1, 1, n), None)
    # tests/test_cf90.F90:9-89: bounded 32^3 (periodic = .FALSE.), dx = 2 pi/31,
    # omega = 12, f = cos(12x) cos(12y) cos(12z), filter1/2/3 (closures 0, 0)
    # against TF(omega dx) f
    n, w = 32, 12.0
    dx = two_pi / (n - 1)
    x, y, z = _axes(n, n, n, dx, dx, dx)
    f = _full(np.cos(w * x) * np.cos(w * y) * np.cos(w * z), sh)
    tf = mod_wavenumber(CF90, FILTER, w, dx)
    lines = {1: "77-79", 2: "82-84", 3: "93-95"}
    for axis in (1, 2, 3):
        yield Check(f"test_cf90:filter{axis}", f"tests/test_cf90.F90:{lines[axis]}", CF90, FILTER, axis, n, 1.0,
                    False, (0, 0), f, tf * f, None)
    if not large:
        return
    # tests/test_filters.F90:50-131 (method 1, cf90): periodic 256^3, dx = 2 pi/256,
    # f = cos x cos y cos z; prints MAXVAL(df - TF f)
    n = 256
    dx = two_pi / n
    x, y, z = _axes(n, n, n, dx, dx, dx)
    sh = (n, n, n)
    f = _full(np.cos(x) * np.cos(y) * np.cos(z), sh)
    tf = mod_wavenumber(CF90, FILTER, 1.0, dx)
    lines = {1: "119-121", 2: "124-126", 3: "129-131"}
    for axis in (1, 2, 3):
        e = tf * f
        yield Check(f"test_filters:filter{axis}", f"tests/test_filters.F90:{lines[axis]}", CF90, FILTER, axis, n,
                    1.0, True, (0, 0), f, e, e, signed=True)
    del f, e
    # tests/test_filters_NP.F90:50-185 (method 1, cf90): bounded 256^3, dx = 2 pi/255,
    # f = sin x sin y sin z, closures (-1, -1): f is odd about 0 and about 2 pi, so
    # the antisymmetric closures reproduce TF f exactly; prints MAXVAL(df - TF f)
    dx = two_pi / (n - 1)
    x, y, z = _axes(n, n, n, dx, dx, dx)
    f = _full(np.sin(x) * np.sin(y) * np.sin(z), sh)
    tf = mod_wavenumber(CF90, FILTER, 1.0, dx)
    lines = {1: "119-122", 2: "124-127", 3: "129-132"}
    for axis in (1, 2, 3):
        e = tf * f
        yield Check(f"test_filters_NP:filter{axis}", f"tests/test_filters_NP.F90:{lines[axis]}", CF90, FILTER,
                    axis, n, 1.0, False, (-1, -1), f, e, e, signed=True)


def recipe_errors(apply: Callable[[Check], np.ndarray] = oracle_apply, large: bool = True) -> dict:
    """The error each reference recipe prints, computed through ``apply``."""
    return {c.name: c.printed(apply(c)) for c in reference_recipes(large)}


# Formal polynomial order of the bc = 0 closures (degree reproduced exactly):
# * cd06 d1 and cd10 d1: the node-1 closure alpha = 3, (p, q, r, s) of
#   cd06.F90:20-24 / cd10.F90:34-38 is third order: cubics are exact;
# * cd10 d2: the node-1 closure b1_* (alpha = 11, cd10.F90:81-87) reproduces
#   x^k for k <= 4 (13 - 27 + 15 - 1 + 0 = 0, -27 + 30 - 3 = 0, ... up to
#   -27 + 15*16 - 81 = 12*11), nodes 2 and 3 (b2_*, b3_*) at least as high;
# * cf90: node 2 (b2_alpha90 = 0.4997, b2_a90 + 2 b2_b90 = 1 + 2 b2_alpha90,
#   cf90.F90:27-29) keeps constants and, being symmetric, linears, but not
#   quadratics (2 b2_b90 != 2 b2_alpha90): degree 1.
CLOSURE_ORDER = {(CD06, D1): 3, (CD10, D1): 3, (CD10, D2): 4, (CF90, FILTER): 1}
PIN_OPS = [(CD06, D1), (CD10, D1), (CD10, D2), (CF90, FILTER)]


def _poly_pin(scheme, kind, n, bc1, bcn, rng):
    """A polynomial of the closure order with the parity the non-zero end
    needs, on [0, 2]; returns (dx, f, exact output)."""
    d = CLOSURE_ORDER[(scheme, kind)]
    L = 2.0
    dx = L / (n - 1)
    x = np.arange(n) * dx
    if bc1 != 0:
        e, par = 0.0, bc1
    elif bcn != 0:
        e, par = L, bcn
    else:
        e, par = 1.0, 0
    s = x - e
    powers = [p for p in range(d + 1) if par == 0 or (p % 2 == 0) == (par == 1)]
    coef = rng.uniform(0.5, 1.0, d + 1) * rng.choice([-1.0, 1.0], d + 1)
    f = sum(coef[p] * s ** p for p in powers)
    if kind == D1:
        ex = sum(coef[p] * p * s ** (p - 1) for p in powers if p >= 1) + 0 * x
    elif kind == D2:
        ex = sum(coef[p] * p * (p - 1) * s ** (p - 2) for p in powers if p >= 2) + 0 * x
    else:
        ex = f
    return dx, f, ex


def _mode_pin(scheme, kind, n, bc1, bcn):
    """cos(3x) (even about 0) or sin(3x) (odd about 0) on [0, L], with L = pi
    (same parity at both ends) or pi/2 (opposite parity); returns (dx, f, exact)."""
    k = 3
    L = np.pi if bc1 == bcn else np.pi / 2
    dx = L / (n - 1)
    x = np.arange(n) * dx
    if bc1 == 1:
        f, fp = np.cos(k * x), -np.sin(k * x)
    else:
        f, fp = np.sin(k * x), np.cos(k * x)
    m = mod_wavenumber(scheme, kind, k, dx)
    if kind == D1:
        ex = m * fp
    elif kind == D2:
        ex = -m * f
    else:
        ex = m * f
    return dx, f, ex


def pin_tolerance(c: Check) -> float:
    """Rounding bound of a closed-form pin on a fixed interval: a first
    derivative loses digits in proportion to 1/dx, i.e. n (max(1e-12, 4e-15 n):
    1e-12 up to n = 250), a second derivative in proportion to n^2 (1e-14 n^2,
    1.6e-11 at n = 40), the filter none (1e-12)."""
    if c.kind == D2:
        return 1e-14 * c.n ** 2
    if c.kind == D1:
        return max(1e-12, 4e-15 * c.n)
    return 1e-12


def closure_pins(n: int = 40, lines: int = 3, seed: int = 11) -> Iterator[Check]:
    """Closed-form known answers for every bounded closure pair, along all
    three axes.  cd06 has only its (0, 0) closures (its bc = 1 branch is
    marked incomplete in cd06.F90:289-293 and leaves the interior rows)."""
    rng = np.random.default_rng(seed)
    for (scheme, kind), (bc1, bcn) in itertools.product(PIN_OPS, itertools.product((0, 1, -1), repeat=2)):
        if scheme == CD06 and (bc1, bcn) != (0, 0):
            continue
        if bc1 != 0 and bcn != 0:
            dx, f1, e1 = _mode_pin(scheme, kind, n, bc1, bcn)
            how = "mode"
        else:
            dx, f1, e1 = _poly_pin(scheme, kind, n, bc1, bcn, rng)
            how = "polynomial"
        for axis in (1, 2, 3):
            sh = [lines, lines + 1, lines + 2]
            sh[3 - axis] = n
            bsh = [1, 1, 1]
            bsh[3 - axis] = n
            # scale each line differently so a transposed or shifted line shows
            w = (1.0 + 0.25 * np.arange(np.prod(sh) // n)).reshape([s if s != n else 1 for s in sh])
            f = np.ascontiguousarray(f1.reshape(bsh) * w)
            ex = np.ascontiguousarray(e1.reshape(bsh) * w)
            yield Check(f"pin:{how}:s{scheme}k{kind}:bc{bc1},{bcn}:axis{axis}", "closure order / mirror parity",
                        scheme, kind, axis, n, dx if scheme != CF90 else 1.0, False, (bc1, bcn), f, ex, ex)
