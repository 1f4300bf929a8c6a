"""GPU: the streaming kernel fed by per-element asynchronous copies (variant
6, cp.async into the tile, one mbarrier arrival per thread) -- the automatic
choice for fields the tensor / bulk copies cannot move: an odd extent along
the contiguous axis (odd na for y/z lines, odd n for x lines) or a pointer
that is 8- but not 16-byte aligned.

Checked through the C ABI against the oracle (max|x - r| / max|r| <= 1e-12)
on fields large enough that every persistent CTA runs several tiles (more
tiles than 2 CTAs x 148 SMs), partial tiles included; against the TMA-fed
kernel (variant 4) bit for bit on even fields (the same arithmetic, only the
copies differ); and through the automatic choice on odd and unaligned fields.
"""
import numpy as np
import pytest

import oracle
from tests.fields import na_nb, rel_err
from tests.test_gpu_parity import OPS, _make, _oracle_apply

pytestmark = pytest.mark.gpu

TOL = 1e-12
# odd extents along every contiguous axis; each launch has > 296 tiles of 16 lines
SHAPES = {1: (67, 91, 129), 2: (67, 129, 129), 3: (129, 67, 129)}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _tiles(shape, axis):
    na, nb = na_nb(shape, axis)
    return (na * nb + 15) // 16 if axis == 1 else (na + 15) // 16 * nb


def _apply(torch, op, kind, axis, ft, bc1=0, bcn=0):
    na, nb = na_nb(tuple(ft.shape), axis)
    out = torch.full_like(ft, float("nan"))
    op.apply(kind, axis, ft, out, na, nb, bc1, bcn)
    torch.cuda.synchronize()
    assert op.device_status() == 0
    return out


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_async_stream_matches_oracle(torch_cuda, scheme, kind, periodic):
    torch = torch_cuda
    rng = np.random.default_rng(61 + 7 * scheme + kind + periodic)
    n = 129
    op = _make(scheme, n, 0.3, periodic)
    bcs = [(0, 0)] if periodic or scheme == oracle.CD06 else [(0, 0), (1, -1), (-1, 1)]
    for variant in (6, 0):
        op.set_variant(variant)
        for axis in (1, 2, 3):
            shape = SHAPES[axis]
            assert _tiles(shape, axis) > 296
            f = rng.standard_normal(shape)
            ft = torch.from_numpy(f).cuda()
            na, nb = na_nb(shape, axis)
            plan = op.launch_plan(kind, axis, ft, torch.empty_like(ft), na, nb)
            assert plan["variant"] == 6, plan
            for bc1, bcn in bcs:
                got = _apply(torch, op, kind, axis, ft, bc1, bcn).cpu().numpy()
                ref = _oracle_apply(scheme, kind, axis, f, 0.3, periodic, bc1, bcn)
                assert rel_err(got, ref) <= TOL, (variant, axis, bc1, bcn)


@pytest.mark.parametrize("scheme,kind", OPS)
def test_async_stream_equals_tma_stream(torch_cuda, scheme, kind):
    """Even extents and aligned fields, where both copy paths can run: the
    results are identical bit for bit, periodic and bounded, every axis,
    segments of 32 and 64 rows."""
    torch = torch_cuda
    rng = np.random.default_rng(71 + 3 * scheme + kind)
    for n, shapes in ((128, {1: (40, 50, 128), 2: (40, 128, 96), 3: (128, 40, 96)}),
                      (1024, {1: (4, 6, 1024), 2: (4, 1024, 34), 3: (1024, 4, 34)})):
        for periodic in (True, False):
            op = _make(scheme, n, 0.2, periodic)
            for axis in (1, 2, 3):
                ft = torch.from_numpy(rng.standard_normal(shapes[axis])).cuda()
                outs = []
                for variant in (4, 6):
                    op.set_variant(variant)
                    na, nb = na_nb(tuple(ft.shape), axis)
                    assert op.launch_plan(kind, axis, ft, torch.empty_like(ft), na, nb)["variant"] == variant
                    outs.append(_apply(torch, op, kind, axis, ft))
                assert torch.equal(outs[0], outs[1]), (n, periodic, axis)


@pytest.mark.parametrize("scheme,kind", OPS)
def test_async_stream_unaligned_fields(torch_cuda, scheme, kind):
    """Fields starting 8 bytes past a 16-byte boundary (input, output or
    both), even extents: the automatic choice streams them by per-element
    copies."""
    torch = torch_cuda
    rng = np.random.default_rng(81 + scheme + kind)
    n = 96
    op = _make(scheme, n, 0.25, False)
    shapes = {1: (20, 30, n), 2: (20, n, 64), 3: (n, 20, 64)}
    for axis in (1, 2, 3):
        shape = shapes[axis]
        f = rng.standard_normal(shape)
        ref = _oracle_apply(scheme, kind, axis, f, 0.25, False, 0, 0)
        size = int(np.prod(shape))
        for off_in, off_out in ((1, 0), (0, 1), (1, 1)):
            fin = torch.zeros(size + 1, dtype=torch.float64, device="cuda")[off_in:off_in + size].view(shape)
            fin.copy_(torch.from_numpy(f))
            out = torch.full((size + 1,), float("nan"), dtype=torch.float64, device="cuda")[off_out:off_out + size]
            out = out.view(shape)
            na, nb = na_nb(shape, axis)
            assert op.launch_plan(kind, axis, fin, out, na, nb)["variant"] == 6
            op.apply(kind, axis, fin, out, na, nb)
            torch.cuda.synchronize()
            assert op.device_status() == 0
            assert rel_err(out.cpu().numpy(), ref) <= TOL, (axis, off_in, off_out)
