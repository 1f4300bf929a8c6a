"""GPU: the staggered sixth-order scheme (pado_cd06stagg_*) through the C ABI
against the oracle (oracle/stagg.py, the restatement of
src/derivatives/cd06stagg.F90): every operator, periodic and non-periodic
with every even / odd / one-sided closure combination, real and complex
fields, line counts that leave partial thread blocks; the closed forms of
tests/stagg_cases.py; the error codes.  Tolerance: max|x - r| / max|r| <=
1e-12."""
import itertools

import numpy as np
import pytest

from oracle.stagg import Stagg
from tests.fields import rel_err
from tests.stagg_cases import OPS, parity_cases, periodic_cases, sided_cases

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _gpu(torch, st, name, f):
    """Apply on a (planes, n2, n1) numpy array (real or complex)."""
    nin, nout = st.sizes(name)
    assert f.shape[0] == nin
    ft = torch.from_numpy(np.ascontiguousarray(f)).cuda()
    out = torch.full((nout,) + f.shape[1:], float("nan"), dtype=ft.dtype, device="cuda")
    getattr(st, name)(ft, out, f.shape[2], f.shape[1])
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _oracle(S, name, f):
    if np.iscomplexobj(f):
        return S.apply(name, np.ascontiguousarray(f.real)) + 1j * S.apply(name, np.ascontiguousarray(f.imag))
    return S.apply(name, f)


CLOSURES = [dict(top_even=te, bot_even=be, top_sided=ts, bot_sided=bs)
            for te, be, ts, bs in itertools.product((True, False), repeat=4)]


@pytest.mark.parametrize("n", [8, 33, 256])
def test_stagg_vs_oracle(torch_cuda, n):
    import padeops_b200 as pb

    torch = torch_cuda
    rng = np.random.default_rng(n)
    dz = 1.0 / n
    setups = [dict(periodic=True)] + [dict(periodic=False, **c) for c in CLOSURES]
    for setup in setups:
        S = Stagg(n, dz, **setup)
        st = pb.cd06stagg()
        if setup["periodic"]:
            assert st.init(n, dz) == 0
        else:
            kw = {k: v for k, v in setup.items() if k != "periodic"}
            assert st.init(n, dz, kw["top_even"], kw["bot_even"], kw["top_sided"], kw["bot_sided"]) == 0
        for name in OPS:
            if setup["periodic"] and name in ("ddz_C2C", "ddz_E2E"):
                with pytest.raises(pb.PadoError):
                    st.sizes(name)
                continue
            nin, _ = st.sizes(name)
            for shape in ((nin, 5, 37), (nin, 3, 64)):
                f = rng.standard_normal(shape)
                assert rel_err(_gpu(torch, st, name, f), _oracle(S, name, f)) <= TOL, (setup, name, shape)
            fc = rng.standard_normal((nin, 2, 9)) + 1j * rng.standard_normal((nin, 2, 9))
            got = _gpu(torch, st, name, fc)
            ref = _oracle(S, name, fc)
            assert np.abs(got - ref).max() / np.abs(ref).max() <= TOL, (setup, name, "complex")
        st.destroy()


def test_stagg_closed_forms(torch_cuda):
    """Periodic modes, parity modes of the even / odd closures and polynomials
    of the one-sided closures, computed on the GPU (<= 1e-12; first
    derivatives of polynomials max(1e-12, 4e-15 n))."""
    import padeops_b200 as pb

    torch = torch_cuda
    n = 64
    st = pb.cd06stagg()
    assert st.init(n, 1.0 / n) == 0
    for name, f, ex, m in periodic_cases(n):
        got = _gpu(torch, st, name, np.broadcast_to(f[:, None, None], (len(f), 2, 40)).copy())
        assert rel_err(got[:, 1, 7], ex) <= TOL, (name, m)
    for be, te, dz, name, f, ex in parity_cases(40):
        assert st.init(40, dz, te, be, False, False) == 0
        got = _gpu(torch, st, name, np.broadcast_to(f[:, None, None], (len(f), 1, 33)).copy())
        assert rel_err(got[:, 0, 32], ex) <= TOL, (be, te, name)
    assert st.init(48, 1.0 / 48, True, True, True, True) == 0
    for name, dz, f, ex in sided_cases(48):
        got = _gpu(torch, st, name, np.broadcast_to(f[:, None, None], (len(f), 1, 33)).copy())
        tol = max(TOL, 4e-15 * 48) if name.startswith("ddz") else TOL
        assert rel_err(got[:, 0, 0], ex) <= tol, name


def test_stagg_full_field(torch_cuda):
    """A 256 x 256 x 384 field (one thread per z line, 65536 lines): periodic
    E2C derivative and non-periodic C2E interpolation against the oracle."""
    import padeops_b200 as pb

    torch = torch_cuda
    n = 384
    rng = np.random.default_rng(5)
    for periodic, name in ((True, "ddz_E2C"), (False, "InterpZ_C2E")):
        st = pb.cd06stagg()
        assert (st.init(n, 1.0 / n) if periodic else st.init(n, 1.0 / n, False, True, False, True)) == 0
        S = Stagg(n, 1.0 / n, True) if periodic else Stagg(n, 1.0 / n, False, False, True, False, True)
        nin, _ = st.sizes(name)
        f = rng.standard_normal((nin, 256, 256))
        assert rel_err(_gpu(torch, st, name, f), S.apply(name, f)) <= TOL, name


def test_stagg_errors(torch_cuda):
    import padeops_b200 as pb
    from padeops_b200 import _lib as L

    torch = torch_cuda
    st = pb.cd06stagg()
    assert st.init(4, 0.25) == 21  # PADO_STAGG_E_SHORT, the reference's exit code
    assert b"4 points" in L.lib().pado_strerror(21)
    assert st.init(8, 0.125) == 0
    f = torch.zeros(9 * 4, dtype=torch.float64, device="cuda")
    with pytest.raises(pb.PadoError):
        st.ddz_E2C(f, f[: 8 * 4], 2, 2)  # overlapping input and output
    with pytest.raises(ValueError):
        st.ddz_E2C(f.cpu(), torch.empty(8 * 4, dtype=torch.float64), 2, 2)  # no CPU path
