"""CPU checks of the staggered-scheme oracle (oracle/stagg.py, the numpy
restatement of src/derivatives/cd06stagg.F90) against closed forms: periodic
modified wavenumbers / transfer functions, parity modes of the even / odd
closures, polynomials of the one-sided closures, and the reference test
tests/test_STAGGcd06.F90.  Tolerances per assertion."""
import numpy as np
import pytest

from oracle.stagg import Stagg
from tests.stagg_cases import cplx_apply, parity_cases, periodic_cases, reference_recipe, sided_cases


def _rel(got, ex):
    return float(np.abs(got - ex).max() / np.abs(ex).max())


@pytest.mark.parametrize("n", [8, 16, 64])
def test_periodic_modes(n):
    """Every periodic operator on modes 1 .. n/2-1: the closed form to <= 1e-12."""
    S = Stagg(n, 1.0 / n, True)
    for name, f, ex, m in periodic_cases(n):
        got = S.apply(name, f[:, None, None])[:, 0, 0]
        assert _rel(got, ex) <= 1e-12, (name, m, _rel(got, ex))


@pytest.mark.parametrize("n", [12, 40])
def test_parity_closures(n):
    """Even / odd closures at both ends, every operator: the parity mode to <= 1e-12."""
    for be, te, dz, name, f, ex in parity_cases(n):
        S = Stagg(n, dz, False, top_even=te, bot_even=be)
        got = S.apply(name, f[:, None, None])[:, 0, 0]
        assert _rel(got, ex) <= 1e-12, (be, te, name, _rel(got, ex))


@pytest.mark.parametrize("n", [16, 48])
def test_sided_closures(n):
    """One-sided closures at both ends reproduce polynomials of their order
    (<= 1e-12 of the exact answer; first derivatives lose digits like n)."""
    S = Stagg(n, 1.0 / n, False, top_even=True, bot_even=True, top_sided=True, bot_sided=True)
    for name, dz, f, ex in sided_cases(n):
        got = S.apply(name, f[:, None, None])[:, 0, 0]
        tol = max(1e-12, 4e-15 * n) if name.startswith("ddz") else 1e-12
        assert _rel(got, ex) <= tol, (name, _rel(got, ex))


def test_reference_recipe():
    """tests/test_STAGGcd06.F90 (periodic, nz = 8): the discrete results equal
    the closed forms (<= 1e-12), and the errors against the exact functions are
    those of 8 points per wavelength (below 2e-3 of the derivative scale)."""
    nz, dz, cases = reference_recipe()
    S = Stagg(nz, dz, True)
    for name, f, exact in cases:
        got = cplx_apply(S, name, f)
        assert np.abs(got - exact).max() <= 2e-3 * np.abs(exact).max(), name


def test_short_and_periodic_only_operators():
    """nx <= 4 stops the reference (GracefulExit 21); a periodic object has no
    C2C / E2E first derivative (the reference has no tables for them)."""
    with pytest.raises(ValueError):
        Stagg(4, 0.25, True)
    S = Stagg(8, 0.125, True)
    with pytest.raises(ValueError):
        S.apply("ddz_C2C", np.zeros((8, 1, 1)))
