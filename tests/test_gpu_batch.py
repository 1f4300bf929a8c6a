"""GPU: batched execution (pado_batch_*) of many uneven (field, operator)
items -- the persistent launch, its CUDA-graph replay and the per-item loop --
against the oracle, plus the batch autotuner.  Tolerance: max|x - r| /
max|r| <= 1e-12 per item."""
import numpy as np
import pytest

import oracle
from tests.fields import na_nb, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
DIMS = (32, 48, 64, 96, 128)


def _items(torch, nitems, seed, dims=DIMS):
    """Random uneven workload: shape, scheme, kind, boundary type, closures, axis."""
    import padeops_b200 as pb

    rng = np.random.default_rng(seed)
    items, host = [], []
    for _ in range(nitems):
        shape = tuple(int(v) for v in rng.choice(dims, size=3))
        scheme = int(rng.choice([oracle.CD06, oracle.CD10, oracle.CF90]))
        kind = {oracle.CD06: oracle.D1, oracle.CF90: oracle.FILTER}.get(scheme, int(rng.choice([oracle.D1, oracle.D2])))
        periodic = bool(rng.integers(2))
        axis = int(rng.integers(1, 4))
        n = shape[3 - axis]
        dx = 2 * np.pi / n if periodic else 1.0 / (n - 1)
        bc1, bcn = (0, 0) if periodic else (int(rng.choice([0, 1, -1])), int(rng.choice([0, 1, -1])))
        ibc = (bc1, bcn) if scheme == oracle.CD06 else (0, 0)
        op = {oracle.CD06: pb.cd06, oracle.CD10: pb.cd10, oracle.CF90: pb.cf90}[scheme]()
        ierr = op.init(n, periodic) if scheme == oracle.CF90 else op.init(n, dx, periodic, *ibc)
        assert ierr == 0
        f = rng.standard_normal(shape)
        ft = torch.from_numpy(f).cuda()
        df = torch.full_like(ft, float("nan"))
        items.append((op, kind, axis, ft, df, bc1, bcn))
        host.append((scheme, kind, n, dx, periodic, ibc, bc1, bcn, axis, f))
    return items, host


def _oracle(h):
    scheme, kind, n, dx, periodic, ibc, bc1, bcn, axis, f = h
    o = oracle.OracleOp(scheme, n, dx, periodic, *ibc)
    na, nb = na_nb(f.shape, axis)
    return o.apply(kind, axis, f, na, nb, bc1, bcn).reshape(f.shape)


def _check(torch, items, host):
    torch.cuda.synchronize()
    for (op, kind, axis, ft, df, bc1, bcn), h in zip(items, host):
        got = df.cpu().numpy()
        assert rel_err(got, _oracle(h)) <= TOL, (h[:9], rel_err(got, _oracle(h)))


@pytest.mark.parametrize("mode", ["run", "run_graph", "run_loop"])
def test_batch_parity(mode):
    import torch

    from padeops_b200.batch import Batch

    items, host = _items(torch, 40, seed=5)
    b = Batch(items)
    for _ in range(2):  # the graph mode captures on the first call and replays on the second
        for it in items:
            it[4].fill_(float("nan"))
        getattr(b, mode)()
        _check(torch, items, host)
        if mode != "run_loop":
            assert b.status() == 0
    b.destroy()


@pytest.mark.parametrize("mode", ["run", "run_graph"])
def test_batch_odd_extents(mode):
    """Odd extents along every axis (the persistent launch copies tiles element
    by element, so no extent or alignment rule applies), partial tiles, many
    tiles per CTA."""
    import torch

    from padeops_b200.batch import Batch

    items, host = _items(torch, 40, seed=31, dims=(31, 48, 65, 97, 127))
    b = Batch(items)
    for _ in range(2):
        for it in items:
            it[4].fill_(float("nan"))
        getattr(b, mode)()
        _check(torch, items, host)
        assert b.status() == 0
    b.destroy()


@pytest.mark.parametrize("mode", ["run", "run_graph"])
def test_batch_long_lines(mode):
    """Items whose lines are 1024 points long (segments of 64 rows), every
    scheme, axis and boundary type, mixed with short ones in one batch."""
    import torch

    import padeops_b200 as pb
    from padeops_b200.batch import Batch

    rng = np.random.default_rng(17)
    items, host = [], []
    n = 1024
    for scheme, kind in ((oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2),
                         (oracle.CF90, oracle.FILTER)):
        for periodic in (True, False):
            dx = 2 * np.pi / n if periodic else 1.0 / (n - 1)
            op = {oracle.CD06: pb.cd06, oracle.CD10: pb.cd10, oracle.CF90: pb.cf90}[scheme]()
            assert (op.init(n, periodic) if scheme == oracle.CF90 else op.init(n, dx, periodic, 0, 0)) == 0
            for axis, shape in ((1, (3, 5, n)), (2, (3, n, 8)), (3, (n, 3, 8))):
                bc1, bcn = (0, 0) if periodic or scheme == oracle.CD06 else (1, -1)
                f = rng.standard_normal(shape)
                ft = torch.from_numpy(f).cuda()
                items.append((op, kind, axis, ft, torch.full_like(ft, float("nan")), bc1, bcn))
                host.append((scheme, kind, n, dx, periodic, (0, 0), bc1, bcn, axis, f))
    short, short_host = _items(torch, 8, seed=23)
    items += short
    host += short_host
    b = Batch(items)
    for _ in range(2):
        for it in items:
            it[4].fill_(float("nan"))
        getattr(b, mode)()
        _check(torch, items, host)
    b.destroy()


def test_batch_96_uneven_fields():
    """The 96-field uneven workload shape (dimensions drawn from the configs'
    set, capped at 128 here to keep the oracle quick)."""
    import torch

    from padeops_b200.batch import Batch

    items, host = _items(torch, 96, seed=96)
    b = Batch(items)
    info = b.info()
    assert info["tiles"] > 0 and info["grid"] > 0
    b.run_graph()
    _check(torch, items, host)
    b.destroy()


def test_batch_autotuner_keeps_results():
    import torch

    from padeops_b200.batch import Batch
    from padeops_b200.tune import tune_batch

    items, host = _items(torch, 16, seed=9)
    b = Batch(items)
    lines, per_sm, branches, ms = tune_batch(b, reps=2)
    assert lines in (0, 8, 16, 32) and per_sm in (0, 1, 2) and branches in (0, 2, 4, 8) and ms > 0
    for it in items:
        it[4].fill_(float("nan"))
    b.run()
    _check(torch, items, host)
    for it in items:
        it[4].fill_(float("nan"))
    b.run_graph()
    _check(torch, items, host)
    b.destroy()


@pytest.mark.parametrize("branches", [1, 4])
def test_batch_graph_of_branches(branches):
    """The graph of per-item streaming-kernel launches on concurrent branches."""
    import torch

    from padeops_b200.batch import Batch

    items, host = _items(torch, 30, seed=13)
    b = Batch(items)
    assert b.set_graph_branches(branches) == 0
    for _ in range(2):
        for it in items:
            it[4].fill_(float("nan"))
        b.run_graph()
        _check(torch, items, host)
    b.destroy()


def test_batch_rejects_bad_items():
    import torch

    import padeops_b200 as pb
    from padeops_b200.batch import Batch
    from padeops_b200._lib import PadoError

    op = pb.cd10()
    assert op.init(64, 0.1, True, 0, 0) == 0
    f = torch.zeros((8, 8, 32), dtype=torch.float64, device="cuda")  # x extent 32 != n
    with pytest.raises(PadoError):
        Batch([(op, oracle.D1, 1, f, torch.empty_like(f), 0, 0)])
