"""GPU parity: every operator of the hot path, through the C ABI, against the
oracle (the CPU restatement of the reference) on seeded inputs.

Tolerance: max|x - r| / max|r| <= 1e-12 (FP64, the bar the operator set is
held to), written per assertion below.
"""
import itertools

import numpy as np
import pytest

import oracle
from tests.fields import line_len, na_nb, rel_err, sinusoids, spectrum53

pytestmark = pytest.mark.gpu

TOL = 1e-12
OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]
BCS = list(itertools.product([0, 1, -1], [0, 1, -1]))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _make(scheme, n, dx, periodic, bc1=0, bcn=0):
    import padeops_b200 as pb

    cls = {oracle.CD06: pb.cd06, oracle.CD10: pb.cd10, oracle.CF90: pb.cf90}[scheme]
    op = cls()
    ierr = op.init(n, periodic) if scheme == oracle.CF90 else op.init(n, dx, periodic, bc1, bcn)
    assert ierr == 0
    return op


def _gpu_apply(torch, op, kind, axis, f, bc1, bcn, adjoint=False):
    shape = f.shape
    na, nb = na_nb(shape, axis)
    ft = torch.from_numpy(np.ascontiguousarray(f)).cuda()
    out = torch.full_like(ft, float("nan"))
    op.apply(kind, axis, ft, out, na, nb, bc1, bcn, adjoint=adjoint)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _oracle_apply(scheme, kind, axis, f, dx, periodic, bc1, bcn, init_bc=(0, 0)):
    n = line_len(f.shape, axis)
    ob1, obn = init_bc if scheme == oracle.CD06 else (0, 0)
    o = oracle.OracleOp(scheme, n, dx, periodic, ob1, obn)
    assert o.ierr == 0
    na, nb = na_nb(f.shape, axis)
    return o.apply(kind, axis, f, na, nb, bc1, bcn).reshape(f.shape)


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("axis", [1, 2, 3])
def test_parity_small(torch_cuda, scheme, kind, periodic, axis):
    torch = torch_cuda
    shape = (19, 24, 33)  # (n3, n2, n1): odd and even line lengths
    f = spectrum53(shape, seed=11 + axis)
    n = line_len(shape, axis)
    dx = 2 * np.pi / n if periodic else 1.0 / (n - 1)
    bcs = [(0, 0)] if (periodic or scheme == oracle.CD06) else BCS
    op = _make(scheme, n, dx, periodic)
    for bc1, bcn in bcs:
        got = _gpu_apply(torch, op, kind, axis, f, bc1, bcn)
        ref = _oracle_apply(scheme, kind, axis, f, dx, periodic, bc1, bcn)
        assert np.isfinite(got).all()
        assert rel_err(got, ref) <= TOL, (bc1, bcn, rel_err(got, ref))


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("n", [8, 10, 11, 17, 32, 64, 65, 127, 256, 384, 512, 1000, 1024])
def test_parity_line_lengths(torch_cuda, scheme, kind, n):
    """Ragged and extreme line lengths (minimum sizes, odd, the configs' 1024)."""
    torch = torch_cuda
    if (scheme == oracle.CF90 and n < 10) or (scheme == oracle.CD06 and n < 8):
        pytest.skip("below the scheme's minimum size")
    rng = np.random.default_rng(n)
    for axis in (1, 3):
        shape = (3, 5, n) if axis == 1 else (n, 3, 6)
        f = rng.standard_normal(shape)
        for periodic in (True, False):
            dx = 0.7
            op = _make(scheme, n, dx, periodic)
            for bc1, bcn in ([(0, 0)] if periodic or scheme == oracle.CD06 else [(0, 0), (1, -1), (-1, 1)]):
                got = _gpu_apply(torch, op, kind, axis, f, bc1, bcn)
                ref = _oracle_apply(scheme, kind, axis, f, dx, periodic, bc1, bcn)
                assert rel_err(got, ref) <= TOL, (axis, periodic, bc1, bcn, rel_err(got, ref))


@pytest.mark.parametrize("variant", [1, 2, 3])
@pytest.mark.parametrize("m,lines", [(16, 8), (16, 16), (16, 32), (32, 8), (32, 16), (32, 32), (64, 8)])
def test_parity_tilings(torch_cuda, m, lines, variant):
    """Every kernel variant and segment length / lines-per-CTA the tuner may
    pick gives the oracle's result, along x (tile path) and z (strided paths)."""
    torch = torch_cuda
    n = 256
    for axis, shape in ((1, (6, 7, n)), (3, (n, 5, 37))):
        f = spectrum53(shape, seed=5 + axis)
        for scheme, kind in OPS:
            for periodic in (True, False):
                op = _make(scheme, n, 0.05, periodic)
                op.set_variant(variant)
                try:
                    op.set_tiling(m, lines)
                except Exception:
                    continue  # not a legal shape for this n
                bc = (0, 0) if periodic else (1, -1)
                got = _gpu_apply(torch, op, kind, axis, f, *bc)
                ref = _oracle_apply(scheme, kind, axis, f, 0.05, periodic, *bc)
                assert rel_err(got, ref) <= TOL, (axis, scheme, kind, periodic, rel_err(got, ref))


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_parity_stream(torch_cuda, scheme, kind, periodic):
    """The streaming kernel (TMA-fed persistent CTAs) along every axis: line
    lengths from the minimum to 512, x extents that leave partial tiles."""
    torch = torch_cuda
    rng = np.random.default_rng(77)
    for n in (10, 34, 100, 256, 512):
        for axis, shape in ((1, (3, 7, n)), (2, (5, n, 22)), (3, (n, 4, 18))):
            f = rng.standard_normal(shape)
            op = _make(scheme, n, 0.3, periodic)
            op.set_variant(4)
            for bc1, bcn in ([(0, 0)] if periodic or scheme == oracle.CD06 else [(0, 0), (1, -1), (-1, 1)]):
                got = _gpu_apply(torch, op, kind, axis, f, bc1, bcn)
                ref = _oracle_apply(scheme, kind, axis, f, 0.3, periodic, bc1, bcn)
                assert rel_err(got, ref) <= TOL, (n, axis, bc1, bcn, rel_err(got, ref))
            assert op.device_status() == 0


@pytest.mark.parametrize("m", [16, 32, 64])
def test_parity_stream_tilings(torch_cuda, m):
    """Streaming kernel with each segment length, and n = 1024 (smooth field:
    the one-sided closures cancel heavily, the stencils must round like the
    reference's expressions)."""
    torch = torch_cuda
    for n in (256, 1024):
        for axis, shape in ((1, (2, 3, n)), (3, (n, 3, 40))):
            f = spectrum53(shape, seed=3 + axis)
            for scheme, kind in OPS:
                for periodic in (True, False):
                    op = _make(scheme, n, 0.05, periodic)
                    op.set_variant(4)
                    try:
                        op.set_tiling(m, 0)
                    except Exception:
                        continue  # not a legal shape for this n
                    bc = (0, 0) if periodic else (-1, 1)
                    got = _gpu_apply(torch, op, kind, axis, f, *bc)
                    ref = _oracle_apply(scheme, kind, axis, f, 0.05, periodic, *bc)
                    assert rel_err(got, ref) <= TOL, (n, axis, scheme, kind, periodic, rel_err(got, ref))


def test_config1_cd06_64cube(torch_cuda):
    """cd06 periodic dd1/dd2/dd3 on the 64^3 sum of 8 sinusoids (dx = 2pi/64)."""
    torch = torch_cuda
    n = 64
    f = sinusoids(n, seed=1234)
    dx = 2 * np.pi / n
    op = _make(oracle.CD06, n, dx, True)
    for axis in (1, 2, 3):
        got = _gpu_apply(torch, op, oracle.D1, axis, f, 0, 0)
        ref = _oracle_apply(oracle.CD06, oracle.D1, axis, f, dx, True, 0, 0)
        assert rel_err(got, ref) <= TOL


def test_cd06_bounded_init_closures(torch_cuda):
    """cd06 bounded takes its closures from init; bc = 1 there keeps interior
    bands (the reference's "Incomplete" branch, cd06.F90:288-291)."""
    torch = torch_cuda
    rng = np.random.default_rng(3)
    f = rng.standard_normal((5, 4, 40))
    for ib in [(0, 0), (1, 1), (0, 1), (1, 0)]:
        op = _make(oracle.CD06, 40, 0.1, False, *ib)
        got = _gpu_apply(torch, op, oracle.D1, 1, f, 0, 0)
        ref = _oracle_apply(oracle.CD06, oracle.D1, 1, f, 0.1, False, 0, 0, init_bc=ib)
        assert rel_err(got, ref) <= TOL, ib


def test_n_equals_one(torch_cuda):
    """n == 1: derivatives return zero, the filter returns a copy (cd10.F90:2037, cf90.F90:1028)."""
    torch = torch_cuda
    f = np.random.default_rng(0).standard_normal((4, 3, 1))
    for scheme, kind in OPS:
        op = _make(scheme, 1, 1.0, True)
        got = _gpu_apply(torch, op, kind, 1, f, 0, 0)
        expect = f if kind == oracle.FILTER else np.zeros_like(f)
        assert np.array_equal(got, expect)


def test_errors(torch_cuda):
    import padeops_b200 as pb
    from padeops_b200 import _lib as L

    torch = torch_cuda
    op = _make(oracle.CD10, 16, 0.1, False)
    f = torch.zeros(16 * 4, dtype=torch.float64, device="cuda")
    df = torch.zeros_like(f)
    with pytest.raises(pb.PadoError) as e:
        op.dd1(f, df, 2, 2, 2, 0)
    assert e.value.status == L.E_BC == 324
    with pytest.raises(pb.PadoError) as e:
        op.dd1(f, f, 2, 2)
    assert e.value.status == L.E_ALIAS
    c6 = _make(oracle.CD06, 16, 0.1, True)
    with pytest.raises(pb.PadoError) as e:
        c6.apply(L.D2, 1, f, df, 2, 2)
    assert e.value.status == L.E_UNSUPPORTED
    with pytest.raises(ValueError):
        op.dd1(f.cpu(), df, 2, 2)  # no CPU path
    assert pb.cd06().init(5, 0.1, True, 0, 0) == 3
    assert pb.cd06().init(7, 0.1, False, 0, 0) == 2
    assert pb.cd10().init(7, 0.1, True, 0, 0) == 2
    assert pb.cf90().init(9, True) == 7


def test_launch_count_and_library(torch_cuda):
    """The CUDA library is what runs: launches are counted by the extension."""
    import padeops_b200 as pb

    torch = torch_cuda
    before = pb.launch_count()
    op = _make(oracle.CD10, 32, 0.1, True)
    f = torch.randn(32 * 9, dtype=torch.float64, device="cuda")
    df = torch.empty_like(f)
    op.dd2(f, df, 3, 3)
    torch.cuda.synchronize()
    assert pb.launch_count() == before + 1


def test_parity_golden_fixtures(torch_cuda):
    """The committed fixtures (tests/golden/oracle_small.npz, written by
    tests/golden/make_golden.py): every operator, both boundary kinds, every
    closure pair along x (cd06 with its closures fixed at init) and all axes."""
    import json
    import os

    torch = torch_cuda
    data = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_small.npz"))
    cases = json.loads(str(data["cases"]))
    for i, c in enumerate(cases):
        op = _make(c["scheme"], c["n"], c["dx"], c["periodic"], c["ibc1"], c["ibcn"])
        got = _gpu_apply(torch, op, c["kind"], c["axis"], data[f"f{i}"], c["bc1"], c["bcn"])
        ref = data[f"df{i}"]
        assert rel_err(got, ref) <= TOL, (c, rel_err(got, ref))


@pytest.mark.parametrize("axis", [1, 2, 3])
def test_apply_host_pipeline(torch_cuda, axis):
    """pado_apply_host splits a field into chunks of whole lines (strided 2-D
    copies for z lines) and overlaps the copies with the solves: the result
    equals the device-resident apply (<= 1e-12), for pinned and pageable host
    memory and for fields that split into uneven chunks."""
    torch = torch_cuda
    rng = np.random.default_rng(40 + axis)
    for shape in ((200, 300, 150), (64, 48, 40), {1: (1, 1, 64), 2: (3, 64, 5), 3: (64, 3, 5)}[axis]):
        n = line_len(shape, axis)
        na, nb = na_nb(shape, axis)
        f = rng.standard_normal(shape)
        for scheme, kind in OPS:
            op = _make(scheme, n, 0.3, True)
            ref = _gpu_apply(torch, op, kind, axis, f, 0, 0)
            pinned = torch.from_numpy(f).pin_memory()
            out = torch.full(shape, float("nan"), dtype=torch.float64).pin_memory()
            op.apply_host(kind, axis, pinned, out, na, nb)
            assert rel_err(out.numpy(), ref) <= TOL, (shape, scheme, kind)
            out2 = np.full(shape, np.nan)
            op.apply_host(kind, axis, f, out2, na, nb)
            assert rel_err(out2, ref) <= TOL, (shape, scheme, kind, "pageable")


def test_bounded_config_full_size(torch_cuda):
    """The bounded workload at its full size, 1024 x 512 x 256 (x, y periodic; z
    bounded, dz = 1/255): f = P3(z) + 0.1 sin(kx x + ky y), seeded.  Checked
    through properties that hold at any size: the bounded cd06 and cd10 first
    derivatives along z reproduce P3'(z) (their closures are exact for cubics),
    and the periodic cd10 first derivatives along x and y equal the modified
    wavenumber times the sine's derivative (<= 1e-11 relative)."""
    from tests.recipes import mod_wavenumber

    torch = torch_cuda
    n1, n2, n3 = 1024, 512, 256
    rng = np.random.default_rng(3)
    c = rng.uniform(-1, 1, 4)
    kx, ky = (int(v) for v in rng.integers(1, 33, 2))
    dx, dy, dz = 2 * np.pi / n1, 2 * np.pi / n2, 1.0 / (n3 - 1)
    x = torch.arange(n1, dtype=torch.float64, device="cuda") * dx
    y = torch.arange(n2, dtype=torch.float64, device="cuda") * dy
    z = torch.arange(n3, dtype=torch.float64, device="cuda") * dz
    phase = kx * x[None, None, :] + ky * y[None, :, None]
    f = (c[0] + c[1] * z + c[2] * z ** 2 + c[3] * z ** 3)[:, None, None] + 0.1 * torch.sin(phase)
    f = f.contiguous()
    df = torch.empty_like(f)
    dp3 = (c[1] + 2 * c[2] * z + 3 * c[3] * z ** 2)[:, None, None].expand(n3, n2, n1)

    def rel(a, b):
        return float((a - b).abs().max() / b.abs().max())

    for scheme in (oracle.CD06, oracle.CD10):
        op = _make(scheme, n3, dz, False)
        op.apply(oracle.D1, 3, f, df, n1, n2, 0, 0)
        torch.cuda.synchronize()
        assert rel(df, dp3) <= 1e-11, (scheme, rel(df, dp3))
    cos = 0.1 * torch.cos(phase).expand(n3, n2, n1)
    for axis, n, d, k in ((1, n1, dx, kx), (2, n2, dy, ky)):
        op = _make(oracle.CD10, n, d, True)
        na, nb = na_nb((n3, n2, n1), axis)
        op.apply(oracle.D1, axis, f, df, na, nb, 0, 0)
        torch.cuda.synchronize()
        ref = mod_wavenumber(oracle.CD10, oracle.D1, k, d) * cos
        assert rel(df, ref) <= 1e-11, (axis, rel(df, ref))


def test_complex_z_filter(torch_cuda):
    """cf90 filter3 on complex fields (filter3_CMPLX) through pado_filter3_complex:
    every closure pair on the right-hand side, the bc (0,0) solve, against the
    oracle (<= 1e-12); a periodic object is refused; n == 1 copies."""
    import padeops_b200 as pb
    from padeops_b200._lib import PadoError

    torch = torch_cuda
    rng = np.random.default_rng(77)
    for n, na, nb in ((10, 3, 2), (33, 8, 5), (256, 20, 6)):
        f = rng.standard_normal((n, nb, na)) + 1j * rng.standard_normal((n, nb, na))
        o = oracle.OracleOp(oracle.CF90, n, 1.0, False)
        op = pb.cf90()
        assert op.init(n, False) == 0
        ft = torch.from_numpy(f).cuda()
        for bc1, bcn in BCS:
            out = torch.full_like(ft, complex(float("nan"), float("nan")))
            op.filter3(ft, out, na, nb, bc1, bcn)
            torch.cuda.synchronize()
            ref = o.filter3_complex(f, na, nb, bc1, bcn).reshape(f.shape)
            got = out.cpu().numpy()
            assert np.abs(got - ref).max() / np.abs(ref).max() <= TOL, (n, bc1, bcn)
    per = pb.cf90()
    assert per.init(64, True) == 0
    ft = torch.zeros((64, 2, 2), dtype=torch.complex128, device="cuda")
    with pytest.raises(PadoError):
        per.filter3(ft, torch.empty_like(ft), 2, 2)
    one = pb.cf90()
    assert one.init(1, True) == 0
    ft = torch.from_numpy(rng.standard_normal((1, 2, 3)) + 1j).cuda()
    out = torch.empty_like(ft)
    one.filter3(ft, out, 3, 2)
    torch.cuda.synchronize()
    assert torch.equal(out, ft)


def test_field_operators(torch_cuda):
    """gradient / curl / divergence / filter3D (operators.F90 counterparts) against
    the same compositions of oracle operators: cd10 periodic x and y, cd06 bounded
    z (closures from init), cf90 periodic x, y and bounded z; numtimes = 2."""
    import padeops_b200 as pb
    from padeops_b200 import field_ops

    torch = torch_cuda
    n1, n2, n3 = 24, 20, 18
    shape = (n3, n2, n1)
    rng = np.random.default_rng(11)
    u, v, w = (rng.standard_normal(shape) for _ in range(3))
    dx, dy, dz = 2 * np.pi / n1, 2 * np.pi / n2, 1.0 / (n3 - 1)
    der = pb.Derivatives()
    der.init(n1, n2, n3, dx, dy, dz, True, True, False, "cd10", "cd10", "cd06")
    fil = pb.Filters()
    fil.init(n1, n2, n3, "cf90", "cf90", "cf90", True, True, False)

    def od(axis, f, bc=(0, 0)):
        scheme, n, d, per = {1: (oracle.CD10, n1, dx, True), 2: (oracle.CD10, n2, dy, True),
                             3: (oracle.CD06, n3, dz, False)}[axis]
        return _oracle_apply(scheme, oracle.D1, axis, f, d, per, *bc)

    def ofil(axis, f, bc=(0, 0)):
        per = axis != 3
        return _oracle_apply(oracle.CF90, oracle.FILTER, axis, f, 1.0, per, *bc)

    T = lambda a: torch.from_numpy(a).cuda()
    gx, gy, gz = (torch.empty(shape, dtype=torch.float64, device="cuda") for _ in range(3))
    field_ops.gradient(der, T(u), gx, gy, gz)
    for got, axis in ((gx, 1), (gy, 2), (gz, 3)):
        assert rel_err(got.cpu().numpy(), od(axis, u)) <= TOL
    cu = torch.empty((3,) + shape, dtype=torch.float64, device="cuda")
    field_ops.curl(der, T(u), T(v), T(w), cu)
    ref = [od(2, w) - od(3, v), od(3, u) - od(1, w), od(1, v) - od(2, u)]
    for k in range(3):
        assert rel_err(cu[k].cpu().numpy(), ref[k]) <= TOL, k
    div = torch.empty(shape, dtype=torch.float64, device="cuda")
    field_ops.divergence(der, T(u), T(v), T(w), div)
    assert rel_err(div.cpu().numpy(), od(1, u) + od(2, v) + od(3, w)) <= TOL
    arr = T(u).clone()
    field_ops.filter3d(fil, arr, numtimes=2, z_bc=(1, -1))
    ref = u
    for axis, bc in ((2, (0, 0)), (1, (0, 0)), (3, (1, -1))):
        for _ in range(2):
            ref = ofil(axis, ref, bc)
    assert rel_err(arr.cpu().numpy(), ref) <= TOL


@pytest.mark.parametrize("scheme,kind", OPS)
def test_parity_resident_plain_loads(torch_cuda, scheme, kind):
    """Variant 5 -- the resident tiles fed by plain loads -- and the automatic
    choice, which streams fields the tensor copies cannot move (odd extents,
    unaligned pointers) by per-element asynchronous copies (variant 6), against
    the oracle: every axis, periodic and bounded, odd and even extents, segments
    of 16, 32 and 64 rows, and an unaligned field."""
    torch = torch_cuda
    rng = np.random.default_rng(5 + scheme)
    for n, shape_of in ((33, lambda n: {1: (5, 7, n), 2: (5, n, 9), 3: (n, 7, 9)}),
                        (256, lambda n: {1: (3, 4, n), 2: (3, n, 38), 3: (n, 3, 37)}),
                        (1024, lambda n: {1: (3, 4, n), 2: (3, n, 7), 3: (n, 3, 7)})):  # 64-row segments
        for periodic in (True, False):
            op = _make(scheme, n, 0.4, periodic)
            for variant in (5, 0):
                op.set_variant(variant)
                for axis in (1, 2, 3):
                    shape = shape_of(n)[axis]
                    f = rng.standard_normal(shape)
                    for bc1, bcn in ([(0, 0)] if periodic or scheme == oracle.CD06 else [(0, 0), (1, -1)]):
                        got = _gpu_apply(torch, op, kind, axis, f, bc1, bcn)
                        ref = _oracle_apply(scheme, kind, axis, f, 0.4, periodic, bc1, bcn)
                        assert rel_err(got, ref) <= TOL, (n, periodic, variant, axis, bc1, bcn)
            # an unaligned (odd-offset) field: the automatic choice cannot use TMA
            op.set_variant(0)
            shape = (3, 4, n)
            f = rng.standard_normal(shape)
            buf = torch.zeros(f.size + 1, dtype=torch.float64, device="cuda")
            ft = buf[1:].view(shape)
            ft.copy_(torch.from_numpy(f))
            out = torch.full((f.size + 1,), float("nan"), dtype=torch.float64, device="cuda")[1:].view(shape)
            na, nb = na_nb(shape, 1)
            op.apply(kind, 1, ft, out, na, nb)
            torch.cuda.synchronize()
            ref = _oracle_apply(scheme, kind, 1, f, 0.4, periodic, 0, 0)
            assert rel_err(out.cpu().numpy(), ref) <= TOL


def test_one_handle_on_two_streams(torch_cuda):
    """A handle is immutable after init: the same operator applied to two
    fields on two CUDA streams at once gives each its own correct result."""
    torch = torch_cuda
    n = 256
    rng = np.random.default_rng(21)
    shape = (n, 8, 64)
    fa, fb = rng.standard_normal(shape), rng.standard_normal(shape)
    op = _make(oracle.CD10, n, 0.05, True)
    ta, tb = torch.from_numpy(fa).cuda(), torch.from_numpy(fb).cuda()
    oa, ob = torch.empty_like(ta), torch.empty_like(tb)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    na, nb = na_nb(shape, 3)
    torch.cuda.synchronize()
    for _ in range(3):
        with torch.cuda.stream(s1):
            op.apply(oracle.D1, 3, ta, oa, na, nb)
        with torch.cuda.stream(s2):
            op.apply(oracle.D1, 3, tb, ob, na, nb)
    torch.cuda.synchronize()
    assert rel_err(oa.cpu().numpy(), _oracle_apply(oracle.CD10, oracle.D1, 3, fa, 0.05, True, 0, 0)) <= TOL
    assert rel_err(ob.cpu().numpy(), _oracle_apply(oracle.CD10, oracle.D1, 3, fb, 0.05, True, 0, 0)) <= TOL
    assert op.device_status() == 0
