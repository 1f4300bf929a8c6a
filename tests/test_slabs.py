"""Distributed-field mode on the host (padeops_b200/slabs.py): the z-slab /
y-slab decomposition, its two transposes, and the distributed operators
against the whole-field oracle -- with the ranks emulated in host threads and
as two gloo processes.  The operator objects here are oracle stand-ins with
the apply() signature of the library's schemes: this checks the data
movement and the decomposition's arithmetic; the GPU test runs the CUDA
operators through the same code.  Tolerance for operator results: max|x -
r| / max|r| <= 1e-12."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
from tests.fields import rel_err

TOL = 1e-12
SHAPES = [(12, 10, 9), (7, 5, 16), (5, 3, 8)]  # n3 and n2 not multiples of the rank count; more ranks than rows


class OracleScheme:
    """The oracle behind the library's apply() signature (host tensors)."""

    def __init__(self, scheme, n, dx, periodic):
        self.o = oracle.OracleOp(scheme, n, dx, periodic)

    def apply(self, kind, axis, f, df, na, nb, bc1=0, bcn=0, alpha=1.0, beta=0.0):
        r = torch.from_numpy(self.o.apply(kind, axis, f.numpy(), na, nb, bc1, bcn)).view(f.shape)
        if beta == 0.0:
            df.copy_(alpha * r if alpha != 1.0 else r)
        else:
            df.add_(r, alpha=alpha)


class OracleDer:
    def __init__(self, shape, periodic):
        n3, n2, n1 = shape
        self.ops = [OracleScheme(oracle.CD10, n, 0.3, periodic) for n in (n1, n2, n3)]


def _whole(shape, seed):
    return torch.from_numpy(np.random.default_rng(seed).standard_normal(shape))


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("size", [1, 2, 3, 4])
def test_decomposition_covers_the_field(shape, size):
    from padeops_b200.slabs import Slabs

    s = [Slabs(shape, size, r) for r in range(size)]
    z = [x.z_range() for x in s]
    y = [x.y_range() for x in s]
    assert z[0][0] == 0 and z[-1][1] == shape[0] and all(a[1] == b[0] for a, b in zip(z, z[1:]))
    assert y[0][0] == 0 and y[-1][1] == shape[1] and all(a[1] == b[0] for a, b in zip(y, y[1:]))
    assert max(b - a for a, b in z) - min(b - a for a, b in z) <= 1


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("size", [2, 3, 4])
def test_transposes_emulated_ranks(shape, size):
    from padeops_b200.slabs import Slabs, run_local, transpose_y_to_z, transpose_z_to_y

    g = _whole(shape, 1)

    def rank(r, ex):
        s = Slabs(shape, size, r)
        fy = transpose_z_to_y(s, s.scatter(g), ex)
        y0, y1 = s.y_range()
        assert torch.equal(fy, g[:, y0:y1, :])
        back = transpose_y_to_z(s, fy.contiguous(), ex)
        assert torch.equal(back, s.scatter(g))
        return True

    assert all(run_local(size, rank))


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("size", [2, 3])
def test_distributed_operators_match_whole_field(periodic, size):
    """Every axis through slabs.apply, and the distributed gradient and
    laplacian, against the oracle on the whole field."""
    from padeops_b200 import _lib as L
    from padeops_b200 import slabs as S

    shape = (16, 12, 10)
    g = _whole(shape, 2)
    der = OracleDer(shape, periodic)
    n3, n2, n1 = shape
    whole = {}
    for axis in (1, 2, 3):
        na, nb = {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]
        for kind in (L.D1, L.D2):
            out = torch.empty_like(g)
            der.ops[axis - 1].apply(kind, axis, g, out, na, nb)
            whole[(axis, kind)] = out

    def rank(r, ex):
        s = S.Slabs(shape, size, r)
        fz = s.scatter(g)
        z0, z1 = s.z_range()
        for axis in (1, 2, 3):
            for kind in (L.D1, L.D2):
                d = torch.full_like(fz, float("nan"))
                S.apply(s, der.ops[axis - 1], kind, axis, fz, d, ex)
                assert rel_err(d.numpy(), whole[(axis, kind)][z0:z1].numpy()) <= TOL, (axis, kind)
        gx, gy, gz = (torch.empty_like(fz) for _ in range(3))
        S.gradient(s, der, fz, gx, gy, gz, ex)
        for got, axis in ((gx, 1), (gy, 2), (gz, 3)):
            assert rel_err(got.numpy(), whole[(axis, L.D1)][z0:z1].numpy()) <= TOL
        lap = torch.empty_like(fz)
        S.laplacian(s, der, fz, lap, ex)
        ref = whole[(2, L.D2)] + whole[(1, L.D2)] + whole[(3, L.D2)]
        assert rel_err(lap.numpy(), ref[z0:z1].numpy()) <= TOL
        return True

    assert all(S.run_local(size, rank))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from padeops_b200 import _lib as L
    from padeops_b200 import dist as pdist
    from padeops_b200 import slabs as S

    d = pdist.init("gloo", timeout_s=60)
    try:
        shape = (11, 9, 8)
        g = _whole(shape, 3)
        s = S.Slabs(shape, world, rank)
        ex = S.dist_exchange(d)
        fz = s.scatter(g)
        fy = S.transpose_z_to_y(s, fz, ex)
        y0, y1 = s.y_range()
        ok = torch.equal(fy, g[:, y0:y1, :]) and torch.equal(S.transpose_y_to_z(s, fy.contiguous(), ex), fz)
        der = OracleDer(shape, True)
        dz = torch.empty_like(fz)
        S.apply(s, der.ops[2], L.D1, 3, fz, dz, ex)
        ref = torch.empty_like(g)
        der.ops[2].apply(L.D1, 3, g, ref, shape[2], shape[1])
        z0, z1 = s.z_range()
        q.put((rank, ok, rel_err(dz.numpy(), ref[z0:z1].numpy())))
        d.barrier()
    finally:
        d.destroy_process_group()


def test_two_gloo_ranks_transpose_and_apply():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    for _ in range(world):
        rank, ok, err = q.get(timeout=10)
        assert ok, rank
        assert err <= TOL, (rank, err)


def test_bad_slab_shape_is_refused():
    from padeops_b200.slabs import LocalExchange, Slabs, transpose_z_to_y

    s = Slabs((4, 4, 4), 2, 0)
    with pytest.raises(ValueError):
        transpose_z_to_y(s, torch.zeros(3, 4, 4, dtype=torch.float64), LocalExchange(2).for_rank(0))
    with pytest.raises(ValueError):
        Slabs((4, 4, 4), 2, 2)
