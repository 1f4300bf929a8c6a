"""CPU checks of the oracle, the C restatement of the reference (oracle/).

The reference ships no golden vectors (its tests print errors and assert
nothing), so the restatement is pinned by:

* the reference's own closed forms: on a periodic grid the discrete
  operators act on a Fourier mode exactly as the modified wavenumber /
  transfer function of src/utilities/spectral.F90:938-1010 predicts;
* an independent dense assembly of the same operators (oracle/dense.py),
  bounded closures and all boundary specifications included;
* replays of the reference tests as written (tests/test_cd06.F90,
  test_cd10.F90, test_cd10_NP.F90, test_cd10_der2.F90, test_cf90.F90,
  test_filters.F90, test_filters_NP.F90): same sizes, grids, functions,
  closures and printed errors; where the discrete answer is known in closed
  form (periodic modes, modes with the parity of symmetric / antisymmetric
  closures) it is checked to rounding, and the other printed errors are
  recorded in tests/golden/recipes.json;
* closed-form known answers for every bounded closure pair: polynomials up to
  each closure's formal order and boundary-parity Fourier modes are
  reproduced exactly, and a planted 1e-7 error in any closure coefficient of
  the dense transcription breaks them;
* the init error codes of the reference (cd06.F90:153-183,
  cd10.F90:219-309, cf90.F90:123-168) and the n == 1 cases.

Tolerances are written per assertion.
"""
import itertools
import json
import os

import numpy as np
import pytest

import oracle
from oracle import dense
from tests.fields import na_nb, rel_err
from tests.recipes import closure_pins, mod_wavenumber, oracle_apply, pin_tolerance, reference_recipes

OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("n", [32, 64])
def test_modified_wavenumber(scheme, kind, n):
    """Single Fourier modes along each axis: result = closed form x mode
    (max error / max |exact| <= 1e-12; the filter's against max |input|)."""
    dx = 2 * np.pi / n
    x = np.arange(n) * dx
    o = oracle.OracleOp(scheme, n, dx, True)
    for k in (1, 3, n // 4, n // 2 - 1):
        f1 = np.sin(k * x + 0.3)
        kp = mod_wavenumber(scheme, kind, k, dx)
        if kind == oracle.D1:
            exact = kp * np.cos(k * x + 0.3)
        elif kind == oracle.D2:
            exact = -kp * f1
        else:
            exact = kp * f1
        for axis in (1, 2, 3):
            shape = [3, 2, 4]
            shape[3 - axis] = n
            sh = tuple(shape)
            bshape = [1, 1, 1]
            bshape[3 - axis] = n
            f = np.broadcast_to(f1.reshape(bshape), sh).copy()
            ex = np.broadcast_to(exact.reshape(bshape), sh)
            na, nb = na_nb(sh, axis)
            got = o.apply(kind, axis, f, na, nb).reshape(sh)
            # near the grid cutoff the filter's output is ~1e-3 of its input:
            # measure its error against the input's magnitude (1)
            scale = max(np.abs(ex).max(), 1.0 if kind == oracle.FILTER else 0.0)
            err = np.abs(got - ex).max() / scale
            assert err <= 1e-12, (k, axis, err)


def test_config1_sinusoids_cd06():
    """Config 1: cd06 periodic dd1/dd2/dd3 of 8 separable sinusoids on 64^3,
    expected in closed form through the modified wavenumber (<= 1e-12)."""
    n = 64
    dx = 2 * np.pi / n
    rng = np.random.default_rng(1)
    x = np.arange(n) * dx
    f = np.zeros((n, n, n))
    ex = [np.zeros((n, n, n)) for _ in range(3)]
    for _ in range(8):
        kx, ky, kz = rng.integers(1, 17, size=3)
        ph = rng.uniform(0, 2 * np.pi)
        arg = kz * x[:, None, None] + ky * x[None, :, None] + kx * x[None, None, :] + ph
        f += np.sin(arg)
        for i, k in enumerate((kx, ky, kz)):
            ex[i] += mod_wavenumber(oracle.CD06, oracle.D1, k, dx) * np.cos(arg)
    o = oracle.OracleOp(oracle.CD06, n, dx, True)
    for axis in (1, 2, 3):
        got = o.apply(oracle.D1, axis, f, n, n).reshape(f.shape)
        assert rel_err(got, ex[axis - 1]) <= 1e-12, (axis, rel_err(got, ex[axis - 1]))


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", [10, 17, 48])
def test_matches_dense_assembly(scheme, kind, periodic, n):
    """The restated LU / Thomas / penta paths equal A^{-1} B from the dense band
    definitions, every boundary specification (<= 1e-12)."""
    dx = 0.37
    rng = np.random.default_rng(n + 7 * scheme + kind)
    bcs = [(0, 0)] if periodic else list(itertools.product([0, 1, -1], [0, 1, -1]))
    for bc1, bcn in bcs:
        o = oracle.OracleOp(scheme, n, dx, periodic, bc1 if scheme == oracle.CD06 else 0,
                            bcn if scheme == oracle.CD06 else 0)
        D = dense.operator(scheme, kind, n, dx, periodic, bc1, bcn)
        for axis in (1, 3):
            sh = (3, 4, n) if axis == 1 else (n, 4, 3)
            f = rng.standard_normal(sh)
            na, nb = na_nb(sh, axis)
            got = o.apply(kind, axis, f, na, nb, bc1, bcn).reshape(sh)
            assert rel_err(got, dense.apply_axis(D, f, axis)) <= 1e-12, (bc1, bcn, axis)


def test_reference_test_recipes():
    """The reference tests replayed as written.  Where the discrete operator's
    answer is known in closed form (periodic Fourier modes; test_cd10_NP's
    cos x with closures (1, -1); test_filters_NP's sin x with closures
    (-1, -1)) the oracle matches it to <= 1e-12.  Every printed error equals
    what tests/golden/recipes.json recorded (1e-13 absolute + 1e-9 relative):
    for test_cd10_der2 and test_cf90, whose bc (0, 0) closures have truncation
    errors, that record is the pin of the closure rows' values."""
    with open(os.path.join(GOLDEN, "recipes.json")) as fh:
        recorded = json.load(fh)
    seen = set()
    for c in reference_recipes():
        got = oracle_apply(c)
        seen.add(c.name)
        if c.closed is not None:
            assert c.closed_err(got) <= 1e-12, (c.name, c.source, c.closed_err(got))
        err = c.printed(got)
        assert abs(err - recorded[c.name]) <= 1e-13 + 1e-9 * abs(recorded[c.name]), (c.name, err, recorded[c.name])
    assert seen == set(recorded)


@pytest.mark.parametrize("n", [16, 40])
def test_closure_pins(n):
    """Every bounded closure pair of cd10 d1, cd10 d2 and cf90 (cd06: (0, 0)),
    along every axis: polynomials up to the closure's formal order and
    boundary-parity Fourier modes are reproduced exactly (tolerance
    ``pin_tolerance``: 1e-12, or 1e-14 n^2 for second derivatives)."""
    count = 0
    for c in closure_pins(n=n):
        err = c.closed_err(oracle_apply(c))
        assert err <= pin_tolerance(c), (c.name, err)
        count += 1
    assert count == 3 * (1 + 9 + 9 + 9)


# closure coefficients of the dense transcription, per operator; the row
# weights w1..w4 are left out (they scale both sides of a row and cancel), as
# are the interior constants the closures are derived from at import time
_PLANT = [("_c6", (oracle.CD06, oracle.D1), ["alpha", "p", "q", "r", "s", "qp", "ap", "app", "qpp", "rpp"]),
          ("_k", (oracle.CD10, oracle.D1), ["alpha", "p", "q", "r", "s", "qp", "ap", "appp", "bppp", "qppp", "rppp",
                                            "sppp", "app", "bpp", "qpp", "rpp"]),
          ("_d2b", (oracle.CD10, oracle.D2), ["a1", "b1", "c1", "d1", "al1", "al2", "a2", "al3", "be3", "a3", "b3"]),
          ("CF2", (oracle.CF90, oracle.FILTER), ["al", "a", "b"]),
          ("CF3", (oracle.CF90, oracle.FILTER), ["al", "be", "a", "b", "c"]),
          ("CF4", (oracle.CF90, oracle.FILTER), ["al", "be", "a", "b", "c", "d"])]


@pytest.mark.parametrize("table,op,keys", _PLANT, ids=[p[0] for p in _PLANT])
def test_pins_catch_planted_closure_errors(table, op, keys, monkeypatch):
    """The closure pins are discriminating: a relative error of 1e-7 planted in
    any closure coefficient of the dense transcription (oracle/dense.py) makes
    them fail by more than 10x their tolerance."""
    checks = [c for c in closure_pins(n=40) if (c.scheme, c.kind) == op and c.axis == 1]

    def worst():
        w = 0.0
        for c in checks:
            D = dense.operator(c.scheme, c.kind, c.n, c.dx, c.periodic, *c.bc)
            w = max(w, c.closed_err(dense.apply_axis(D, c.f, c.axis)) / pin_tolerance(c))
        return w

    assert worst() <= 1.0
    d = getattr(dense, table)
    for key in keys:
        with monkeypatch.context() as m:
            m.setitem(d, key, d[key] * (1 + 1e-7))
            assert worst() > 10.0, (table, key)


def test_init_errors_and_n1():
    """init status codes of the reference (too-short lines) and n == 1."""
    assert oracle.OracleOp(oracle.CD06, 5, 0.1, True).ierr == 3    # cd06.F90:153-160
    assert oracle.OracleOp(oracle.CD06, 7, 0.1, False).ierr == 2   # cd06.F90:161-168
    assert oracle.OracleOp(oracle.CD10, 7, 0.1, True).ierr == 2    # cd10.F90:219-230
    assert oracle.OracleOp(oracle.CF90, 9, 1.0, True).ierr == 7    # cf90.F90:123-130
    for scheme, kind in OPS:
        o = oracle.OracleOp(scheme, 1, 1.0, True)
        assert o.ierr == 0
        f = np.arange(6.0) + 1
        got = o.apply(kind, 1, f, 3, 2)
        # n == 1: derivatives are zero, the filter copies (cd06.F90:781-784, cd10.F90:2037-2040, cf90.F90:1028-1031)
        assert np.array_equal(got, f if kind == oracle.FILTER else np.zeros_like(f))


def test_bad_boundary_specification():
    """bc outside {0, 1, -1}: the reference stops with code 324 (cd10.F90:2042-2058)."""
    o = oracle.OracleOp(oracle.CD10, 16, 0.1, False)
    f = np.zeros(16 * 4)
    with pytest.raises(RuntimeError, match="324"):
        o.apply(oracle.D1, 1, f, 2, 2, 2, 0)


def test_golden_fixtures():
    """The committed oracle outputs (tests/golden/oracle_small.npz) are reproduced
    bit for bit: the restatement has not drifted since they were made."""
    data = np.load(os.path.join(GOLDEN, "oracle_small.npz"))
    cases = json.loads(str(data["cases"]))
    for i, c in enumerate(cases):
        f = data[f"f{i}"]
        o = oracle.OracleOp(c["scheme"], c["n"], c["dx"], c["periodic"], c["ibc1"], c["ibcn"])
        na, nb = na_nb(f.shape, c["axis"])
        got = o.apply(c["kind"], c["axis"], f, na, nb, c["bc1"], c["bcn"]).reshape(f.shape)
        assert np.array_equal(got, data[f"df{i}"]), c


def test_complex_z_filter():
    """filter3_CMPLX (cf90.F90:1230-1251): the real and imaginary parts are
    filtered alone, the right-hand side with the closures (bc1, bcn) and the
    solve with the bc (0,0) system -- so for bc (0,0) it equals the real
    filter3 of each part, and for other closures it equals A_00^{-1} B_bc."""
    rng = np.random.default_rng(8)
    n, na, nb = 40, 3, 2
    o = oracle.OracleOp(oracle.CF90, n, 1.0, False)
    f = rng.standard_normal((n, nb, na)) + 1j * rng.standard_normal((n, nb, na))
    for bc1, bcn in itertools.product([0, 1, -1], [0, 1, -1]):
        got = o.filter3_complex(f, na, nb, bc1, bcn).reshape(f.shape)
        D = np.linalg.solve(dense.lhs(oracle.CF90, oracle.FILTER, n, False, 0, 0),
                            dense.rhs(oracle.CF90, oracle.FILTER, n, 1.0, False, bc1, bcn))
        ref = dense.apply_axis(D, f.real, 3) + 1j * dense.apply_axis(D, f.imag, 3)
        assert np.abs(got - ref).max() / np.abs(ref).max() <= 1e-12, (bc1, bcn)
        if (bc1, bcn) == (0, 0):
            re = o.apply(oracle.FILTER, 3, np.ascontiguousarray(f.real), na, nb).reshape(f.shape)
            assert np.array_equal(got.real, re)
    with pytest.raises(RuntimeError, match="-3"):
        oracle.OracleOp(oracle.CF90, n, 1.0, True).filter3_complex(f, na, nb)
