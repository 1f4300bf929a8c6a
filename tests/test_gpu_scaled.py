"""GPU: the scaled / accumulating apply (pado_apply_scaled: df = alpha D f +
beta df, beta 0 or 1) through every kernel that can run a forward operator --
the streaming kernel (y/z lines straight from the sweep, x lines through the
tile), its plain-load variant, the line kernels -- and the n == 1 cases,
against the oracle: max|got - (alpha r + beta df0)| / max|alpha r + beta df0|
<= 1e-12.  Plus the laplacian built on it (cgrid.F90:480-517)."""
import numpy as np
import pytest

import oracle
from tests.fields import na_nb, rel_err, spectrum53
from tests.test_gpu_parity import _make, _oracle_apply

pytestmark = pytest.mark.gpu

TOL = 1e-12
OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("variant", [0, 4, 6, 5, 1, 2, 3])
@pytest.mark.parametrize("periodic", [True, False])
def test_scaled_and_accumulated(torch_cuda, variant, periodic):
    torch = torch_cuda
    rng = np.random.default_rng(7 + variant + 10 * periodic)
    for scheme, kind in OPS:
        for n in (48, 49, 256):
            for axis, shape in ((1, (6, 5, n)), (2, (4, n, 21 + n % 2)), (3, (n, 5, 17 + n % 2))):
                f = rng.standard_normal(shape)
                df0 = rng.standard_normal(shape)
                op = _make(scheme, n, 0.2, periodic)
                op.set_variant(variant)
                na, nb = na_nb(shape, axis)
                bc = (0, 0) if periodic or scheme == oracle.CD06 else (1, -1)
                ref = _oracle_apply(scheme, kind, axis, f, 0.2, periodic, *bc)
                ft = torch.from_numpy(f).cuda()
                for alpha, beta in ((1.0, 0.0), (-0.75, 0.0), (1.0, 1.0), (-1.0, 1.0), (2.5, 1.0)):
                    out = torch.from_numpy(df0.copy()).cuda()
                    try:
                        op.apply(kind, axis, ft, out, na, nb, *bc, alpha=alpha, beta=beta)
                    except Exception as exc:  # a variant that cannot take this field
                        if variant in (4, 5):
                            continue
                        raise exc
                    torch.cuda.synchronize()
                    expect = alpha * ref + beta * df0
                    err = rel_err(out.cpu().numpy(), expect)
                    assert err <= TOL, (scheme, kind, n, axis, alpha, beta, err)
                assert op.device_status() == 0


def test_scaled_n_equals_one_and_errors(torch_cuda):
    """n == 1: a derivative adds alpha * 0, the filter alpha * f; beta outside
    {0, 1} and a scaled adjoint are refused."""
    import padeops_b200 as pb

    torch = torch_cuda
    rng = np.random.default_rng(2)
    f = torch.from_numpy(rng.standard_normal((4, 3, 1))).cuda()
    df0 = rng.standard_normal((4, 3, 1))
    for scheme, kind in OPS:
        op = _make(scheme, 1, 1.0, True)
        for alpha, beta in ((3.0, 0.0), (3.0, 1.0)):
            out = torch.from_numpy(df0.copy()).cuda()
            op.apply(kind, 1, f, out, 3, 4, alpha=alpha, beta=beta)
            torch.cuda.synchronize()
            d = f.cpu().numpy() if kind == oracle.FILTER else np.zeros_like(df0)
            assert np.allclose(out.cpu().numpy(), alpha * d + beta * df0, rtol=0, atol=1e-15)
    op = _make(oracle.CD10, 32, 0.1, True)
    g = torch.zeros(32 * 4, dtype=torch.float64, device="cuda")
    with pytest.raises(pb.PadoError):
        op.apply(oracle.D1, 1, g, torch.zeros_like(g), 2, 2, alpha=1.0, beta=0.5)
    with pytest.raises(pb.PadoError):
        op.apply(oracle.D1, 1, g, torch.zeros_like(g), 2, 2, adjoint=True, alpha=2.0)


def test_laplacian_and_divergence_full_field(torch_cuda):
    """laplacian = d2/dy2 + d2/dx2 + d2/dz2 summed in the kernels (cd10 periodic
    x, y; cd10 bounded z with closures (1, -1)) and divergence (negated
    closures), against oracle compositions summed in the same order; 128^3
    fields, so every kernel runs many tiles."""
    import padeops_b200 as pb
    from padeops_b200 import field_ops

    torch = torch_cuda
    n = 128
    shape = (n, n, n)
    u, v, w = (spectrum53(shape, seed=s) for s in (1, 2, 3))
    dx, dz = 2 * np.pi / n, 1.0 / (n - 1)
    der = pb.Derivatives()
    der.init(n, n, n, dx, dx, dz, True, True, False, "cd10", "cd10", "cd10")

    def od(kind, axis, f, bc=(0, 0)):
        d, per = (dz, False) if axis == 3 else (dx, True)
        return _oracle_apply(oracle.CD10, kind, axis, f, d, per, *bc)

    T = lambda a: torch.from_numpy(a).cuda()
    lap = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
    field_ops.laplacian(der, T(u), lap, z_bc=(1, -1))
    ref = od(oracle.D2, 2, u) + od(oracle.D2, 1, u)
    ref = ref + od(oracle.D2, 3, u, (1, -1))
    assert rel_err(lap.cpu().numpy(), ref) <= TOL
    div = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
    field_ops.divergence(der, T(u), T(v), T(w), div, z_bc=(1, -1))
    ref = od(oracle.D1, 2, v) + od(oracle.D1, 1, u)
    ref = ref + od(oracle.D1, 3, w, (-1, 1))
    assert rel_err(div.cpu().numpy(), ref) <= TOL


def test_host_terms(torch_cuda):
    """pado_apply_host_terms: gradient and laplacian of a host field (pinned and
    pageable) equal the device-resident field operators bit for bit; terms out
    of order are refused."""
    import padeops_b200 as pb
    from padeops_b200 import _lib as L
    from padeops_b200 import field_ops

    torch = torch_cuda
    n1, n2, n3 = 96, 80, 64
    shape = (n3, n2, n1)
    f = spectrum53(shape, seed=9)
    der = pb.Derivatives()
    der.init(n1, n2, n3, 2 * np.pi / n1, 2 * np.pi / n2, 1.0 / (n3 - 1), True, True, False, "cd10", "cd10", "cd10")
    ft = torch.from_numpy(f).cuda()
    g = [torch.empty_like(ft) for _ in range(3)]
    field_ops.gradient(der, ft, *g, z_bc=(1, -1))
    lap = torch.empty_like(ft)
    field_ops.laplacian(der, ft, lap, z_bc=(1, -1))
    torch.cuda.synchronize()
    for pinned in (True, False):
        src = torch.from_numpy(f).pin_memory() if pinned else f
        outs = [np.full(shape, np.nan) for _ in range(3)]
        field_ops.gradient_host(der, src, *outs, z_bc=(1, -1))
        for o, ref in zip(outs, g):
            assert np.array_equal(o, ref.cpu().numpy())
        lo = np.full(shape, np.nan)
        field_ops.laplacian_host(der, src, lo, z_bc=(1, -1))
        assert np.array_equal(lo, lap.cpu().numpy())
    with pytest.raises(pb.PadoError):
        field_ops.apply_host_terms(f, shape, [(der.ops[0], L.D1, 1, 0, 0, 1.0, 1.0, 0)], [np.empty(shape)])
