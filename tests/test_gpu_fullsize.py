"""GPU parity at the workloads' full sizes and on the reference tests' recipes.

* the reference tests replayed as written (tests/recipes.py) and the closed-form
  closure pins, through the CUDA path: against the oracle (<= 1e-12) and
  against the closed forms (``pin_tolerance``);
* the 512^3 step the benchmark times -- cd10 d1, cd10 d2 and cf90 along x, y
  and z on the seeded |k|^-5/3 field -- against the oracle (<= 1e-12).  Each
  launch covers 16384 tiles of 16 lines, so every persistent CTA runs many
  tiles (buffer reuse, barrier phases, copy waits) under the check;
* the bounded workload at its full size (1024 x 512 x 256): cd06, cd10 d1,
  cd10 d2 and cf90 along z with every closure pair, periodic cd06 / cd10
  along x and y, against the oracle (<= 1e-12);
* the batched workload of the benchmark (96 fields, dimensions up to 384)
  against the oracle, for the persistent launch and the tuned graph.

The oracle is the strict build (no fast-math) of the C restatement.
"""
import itertools

import numpy as np
import pytest

import oracle
from tests.fields import na_nb, poly_z, rel_err, spectrum53
from tests.recipes import Check, closure_pins, oracle_apply, pin_tolerance, reference_recipes
from tests.test_gpu_parity import _gpu_apply, _make

pytestmark = pytest.mark.gpu

TOL = 1e-12
BCS = list(itertools.product([0, 1, -1], [0, 1, -1]))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _check_gpu(torch, c: Check) -> np.ndarray:
    op = _make(c.scheme, c.n, c.dx, c.periodic, *(c.bc if c.scheme == oracle.CD06 else (0, 0)))
    got = _gpu_apply(torch, op, c.kind, c.axis, c.f, *c.bc)
    assert op.device_status() == 0
    return got


def test_reference_recipes_gpu(torch_cuda):
    """Every reference recipe (test_cd06, test_cd10, test_cd10_NP,
    test_cd10_der2, test_cf90, test_filters, test_filters_NP; 256^3 ones
    included) through the CUDA path: equal to the oracle (<= 1e-12) and, where
    the answer is known in closed form, to it (<= 1e-12)."""
    torch = torch_cuda
    for c in reference_recipes():
        got = _check_gpu(torch, c)
        assert rel_err(got, oracle_apply(c)) <= TOL, (c.name, c.source)
        if c.closed is not None:
            assert c.closed_err(got) <= 1e-12, (c.name, c.closed_err(got))


@pytest.mark.parametrize("n", [40, 200, 1024])
def test_closure_pins_gpu(torch_cuda, n):
    """Closed-form known answers of every bounded closure pair, along every
    axis, through the CUDA path: equal to the oracle (<= 1e-12) and to the
    closed form (``pin_tolerance``)."""
    torch = torch_cuda
    for c in closure_pins(n=n):
        got = _check_gpu(torch, c)
        assert rel_err(got, oracle_apply(c)) <= TOL, c.name
        assert c.closed_err(got) <= pin_tolerance(c), (c.name, c.closed_err(got))


def test_step_512cube_vs_oracle(torch_cuda):
    """The nine operators of the benchmarked 512^3 step (cd10 d1, cd10 d2, cf90;
    periodic; x, y, z) on the benchmark's seeded field, against the oracle."""
    torch = torch_cuda
    n = 512
    f = spectrum53((n, n, n), seed=7)
    ft = torch.from_numpy(f).cuda()
    out = torch.empty_like(ft)
    dx = 2 * np.pi / n
    for scheme, kind in ((oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)):
        op = _make(scheme, n, dx, True)
        o = oracle.OracleOp(scheme, n, dx, True)
        for axis in (1, 2, 3):
            out.fill_(float("nan"))
            op.apply(kind, axis, ft, out, n, n)
            torch.cuda.synchronize()
            assert op.device_status() == 0
            ref = o.apply(kind, axis, f, n, n).reshape(f.shape)
            err = rel_err(out.cpu().numpy(), ref)
            assert err <= TOL, (scheme, kind, axis, err)


def test_bounded_workload_full_size_vs_oracle(torch_cuda):
    """The bounded workload at 1024 x 512 x 256 (f = P3(z) + 0.1 sin(kx x + ky y),
    seeded; dz = 1/255): cd06 (closures (0, 0) from init), cd10 d1, cd10 d2 and
    cf90 along z with every closure pair, and periodic cd06 / cd10 d1 along x
    and y, against the oracle."""
    torch = torch_cuda
    shape = (256, 512, 1024)
    f = poly_z(shape, seed=3)
    ft = torch.from_numpy(f).cuda()
    out = torch.empty_like(ft)
    n3, n2, n1 = shape
    dz = 1.0 / (n3 - 1)
    cases = [(oracle.CD06, oracle.D1, (0, 0))]
    cases += [(oracle.CD10, k, bc) for k in (oracle.D1, oracle.D2) for bc in BCS]
    cases += [(oracle.CF90, oracle.FILTER, bc) for bc in BCS]
    ops = {}
    for scheme, kind, bc in cases:
        if scheme not in ops:
            ops[scheme] = (_make(scheme, n3, dz, False), oracle.OracleOp(scheme, n3, dz if scheme != oracle.CF90 else 1.0,
                                                                           False))
        op, o = ops[scheme]
        out.fill_(float("nan"))
        op.apply(kind, 3, ft, out, n1, n2, *bc)
        torch.cuda.synchronize()
        ref = o.apply(kind, 3, f, n1, n2, *bc).reshape(shape)
        err = rel_err(out.cpu().numpy(), ref)
        assert err <= TOL, (scheme, kind, bc, err)
    for scheme, axis in itertools.product((oracle.CD06, oracle.CD10), (1, 2)):
        n = n1 if axis == 1 else n2
        d = 2 * np.pi / n
        op = _make(scheme, n, d, True)
        na, nb = na_nb(shape, axis)
        out.fill_(float("nan"))
        op.apply(oracle.D1, axis, ft, out, na, nb)
        torch.cuda.synchronize()
        ref = oracle.OracleOp(scheme, n, d, True).apply(oracle.D1, axis, f, na, nb).reshape(shape)
        err = rel_err(out.cpu().numpy(), ref)
        assert err <= TOL, (scheme, axis, err)
        assert op.device_status() == 0


@pytest.mark.parametrize("mode", ["run", "run_graph"])
def test_batch_benchmark_workload_vs_oracle(torch_cuda, mode):
    """The benchmark's batched workload shape: 96 fields with dimensions drawn
    from {32, ..., 384} (total <= 4 GiB), cd06 or cd10 first derivatives,
    periodic or bounded, random axis; seeded normal fields; every item against
    the oracle after the persistent launch or the autotuned graph."""
    import padeops_b200 as pb
    from padeops_b200.batch import Batch
    from padeops_b200.tune import tune_batch

    torch = torch_cuda
    rng = np.random.default_rng(4)
    dims = (32, 48, 64, 96, 128, 192, 256, 384)
    while True:
        shapes = [tuple(int(v) for v in rng.choice(dims, 3)) for _ in range(96)]
        if sum(a * b * c for a, b, c in shapes) * 8 <= 4 * 2 ** 30:
            break
    items, host = [], []
    for sh in shapes:
        scheme, periodic, axis = int(rng.integers(2)), bool(rng.integers(2)), int(rng.integers(1, 4))
        n = sh[3 - axis]
        dx = 2 * np.pi / n if periodic else 1.0 / (n - 1)
        op = (pb.cd06 if scheme == 0 else pb.cd10)()
        assert op.init(n, dx, periodic, 0, 0) == 0
        f = rng.standard_normal(sh)
        ft = torch.from_numpy(f).cuda()
        items.append((op, oracle.D1, axis, ft, torch.full_like(ft, float("nan")), 0, 0))
        host.append((scheme, n, dx, periodic, axis, f))
    b = Batch(items)
    if mode == "run_graph":
        tune_batch(b, reps=2)
    getattr(b, mode)()
    torch.cuda.synchronize()
    for (op, kind, axis, ft, df, _, _), (scheme, n, dx, periodic, axis_, f) in zip(items, host):
        o = oracle.OracleOp(scheme, n, dx, periodic)
        na, nb = na_nb(f.shape, axis)
        ref = o.apply(oracle.D1, axis, f, na, nb).reshape(f.shape)
        assert rel_err(df.cpu().numpy(), ref) <= TOL, (f.shape, scheme, periodic, axis)
    b.destroy()
