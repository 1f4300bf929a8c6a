"""GPU adjoint: pado_apply_adjoint against D^T assembled densely from the
reference operator (oracle/dense.py), and the autograd wrapper against
central finite differences.

Tolerances: adjoint vs dense D^T <= 1e-11 relative (FP64, dense solve in the
check); gradient vs finite differences <= 1e-8 relative.
"""
import itertools

import numpy as np
import pytest

import oracle
from oracle import dense
from tests.fields import line_len, na_nb, rel_err, spectrum53

pytestmark = pytest.mark.gpu

OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]


def _make(scheme, n, dx, periodic):
    import padeops_b200 as pb

    cls = {oracle.CD06: pb.cd06, oracle.CD10: pb.cd10, oracle.CF90: pb.cf90}[scheme]
    op = cls()
    assert (op.init(n, periodic) if scheme == oracle.CF90 else op.init(n, dx, periodic, 0, 0)) == 0
    return op


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", [10, 24, 40, 100])
def test_adjoint_vs_dense(scheme, kind, periodic, n):
    import torch

    rng = np.random.default_rng(n + 7 * scheme)
    dx = 0.3
    op = _make(scheme, n, dx, periodic)
    bcs = [(0, 0)] if (periodic or scheme == oracle.CD06) else list(itertools.product([0, 1, -1], [0, 1, -1]))
    for bc1, bcn in bcs:
        D = dense.operator(scheme, kind, n, dx, periodic, bc1, bcn)
        for axis in (1, 2, 3):
            shape = {1: (3, 4, n), 2: (3, n, 5), 3: (n, 4, 3)}[axis]
            g = rng.standard_normal(shape)
            na, nb = na_nb(shape, axis)
            gt = torch.from_numpy(g).cuda()
            out = torch.empty_like(gt)
            op.apply(kind, axis, gt, out, na, nb, bc1, bcn, adjoint=True)
            torch.cuda.synchronize()
            ref = dense.apply_axis(D.T, g, axis)
            assert rel_err(out.cpu().numpy(), ref) <= 1e-11, (bc1, bcn, axis)


def test_autograd_vs_finite_differences():
    """L = 0.5 ||D_x^cd10 u + D_z^cd06,bounded u - g||^2 on 32^3: gradient from the
    adjoint kernels vs central differences (h = 1e-6) along 16 seeded directions."""
    import torch

    from padeops_b200.autograd import compact_op

    n = 32
    shape = (n, n, n)
    u = torch.from_numpy(spectrum53(shape, 21)).cuda().requires_grad_(True)
    g = torch.from_numpy(spectrum53(shape, 22)).cuda()
    cx = _make(oracle.CD10, n, 2 * np.pi / n, True)
    cz = _make(oracle.CD06, n, 1.0 / (n - 1), False)

    def loss(v):
        r = compact_op(cx, oracle.D1, 1, v) + compact_op(cz, oracle.D1, 3, v) - g
        return 0.5 * (r * r).sum()

    Lv = loss(u)
    (grad,) = torch.autograd.grad(Lv, u)
    rng = np.random.default_rng(99)
    h = 1e-6
    eps = np.finfo(np.float64).eps
    with torch.no_grad():
        for _ in range(16):
            d = torch.from_numpy(rng.standard_normal(shape)).cuda()
            d /= d.norm()
            lp, lm = float(loss(u + h * d)), float(loss(u - h * d))
            fd = (lp - lm) / (2 * h)
            an = float((grad * d).sum())
            # L is quadratic, so central differences carry no truncation error;
            # what is left is the rounding of L(u +- h d), about eps*|L|/h.
            floor = 8 * eps * (abs(lp) + abs(lm)) / (2 * h)
            assert abs(fd - an) <= 1e-8 * abs(an) + floor, (fd, an, floor)


def test_autograd_vs_dense_transpose():
    """The same loss on a 64^3 copy: the gradient equals the one built from the
    dense D^T of the oracle's operators (<= 1e-11 relative)."""
    import torch

    from padeops_b200.autograd import compact_op

    n = 64
    shape = (n, n, n)
    rng = np.random.default_rng(5)
    u0 = rng.standard_normal(shape)
    g0 = rng.standard_normal(shape)
    dxx, dzz = 2 * np.pi / n, 1.0 / (n - 1)
    cx = _make(oracle.CD10, n, dxx, True)
    cz = _make(oracle.CD06, n, dzz, False)
    u = torch.from_numpy(u0).cuda().requires_grad_(True)
    g = torch.from_numpy(g0).cuda()
    r = compact_op(cx, oracle.D1, 1, u) + compact_op(cz, oracle.D1, 3, u) - g
    (0.5 * (r * r).sum()).backward()
    Dx = dense.operator(oracle.CD10, oracle.D1, n, dxx, True)
    Dz = dense.operator(oracle.CD06, oracle.D1, n, dzz, False)
    rr = dense.apply_axis(Dx, u0, 1) + dense.apply_axis(Dz, u0, 3) - g0
    ref = dense.apply_axis(Dx.T, rr, 1) + dense.apply_axis(Dz.T, rr, 3)
    assert rel_err(u.grad.cpu().numpy(), ref) <= 1e-11


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_stream_adjoint_vs_dense(scheme, kind, periodic):
    """The streaming kernel's adjoint (variant 4: transposed sweep in the tile,
    then B^T) against the dense D^T, every axis, lengths with one or many
    segments and partial tiles; the line kernel's adjoint (variant 1) on the
    same inputs agrees too."""
    import torch

    rng = np.random.default_rng(31 + scheme + 5 * kind)
    for n in (10, 34, 100, 256, 512):
        dx = 0.3
        op = _make(scheme, n, dx, periodic)
        bcs = [(0, 0)] if (periodic or scheme == oracle.CD06) else [(0, 0), (1, -1), (-1, 1), (1, 1)]
        for bc1, bcn in bcs:
            D = dense.operator(scheme, kind, n, dx, periodic, bc1, bcn)
            for axis in (1, 2, 3):
                shape = {1: (3, 5, n), 2: (3, n, 38), 3: (n, 3, 22)}[axis]
                g = rng.standard_normal(shape)
                na, nb = na_nb(shape, axis)
                gt = torch.from_numpy(g).cuda()
                ref = dense.apply_axis(D.T, g, axis)
                for variant in (4, 1):
                    op.set_variant(variant)
                    out = torch.full_like(gt, float("nan"))
                    op.apply(kind, axis, gt, out, na, nb, bc1, bcn, adjoint=True)
                    torch.cuda.synchronize()
                    assert op.device_status() == 0
                    assert rel_err(out.cpu().numpy(), ref) <= 1e-11, (n, bc1, bcn, axis, variant)
                op.set_variant(0)


def test_differentiation_workload_256():
    """The differentiation workload: L = 0.5 ||D_x^cd10 u + D_z^cd06,bounded u - g||^2
    on 256^3 (u, g seeded k^-5/3 fields).  The autograd gradient (adjoint kernels)
    against central differences with h = 1e-6 along 64 seeded directions d (unit
    RMS per point, as u):
    [L(u + h d) - L(u - h d)] / 2h from two forward evaluations r+- = D(u +- h d) - g,
    summed as 0.5 sum (r+ - r-)(r+ + r-) so that the difference of two large sums
    does not cancel.  L is quadratic, so the only error left is rounding:
    relative error <= 1e-8 per direction."""
    import torch

    from padeops_b200.autograd import compact_op

    n = 256
    shape = (n, n, n)
    u = torch.from_numpy(spectrum53(shape, 51)).cuda().requires_grad_(True)
    g = torch.from_numpy(spectrum53(shape, 52)).cuda()
    cx = _make(oracle.CD10, n, 2 * np.pi / n, True)
    cz = _make(oracle.CD06, n, 1.0 / (n - 1), False)

    def resid(v):
        return compact_op(cx, oracle.D1, 1, v) + compact_op(cz, oracle.D1, 3, v) - g

    r0 = resid(u)
    (grad,) = torch.autograd.grad(0.5 * (r0 * r0).sum(), u)
    gen = torch.Generator(device="cuda").manual_seed(64)
    h = 1e-6
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            # unit RMS per point, like u: the step h d is 1e-6 of the field
            d = torch.randn(shape, dtype=torch.float64, device="cuda", generator=gen)
            rp, rm = resid(u + h * d), resid(u - h * d)
            fd = float(0.5 * ((rp - rm) * (rp + rm)).sum()) / (2 * h)
            an = float((grad * d).sum())
            worst = max(worst, abs(fd - an) / abs(an))
    assert worst <= 1e-8, worst
