"""GPU: the distributed-field mode (padeops_b200/slabs.py) with the CUDA
operators, its ranks emulated as host threads on one GPU (the exchange is an
in-process all-to-all; no kernel waits on another).  Each rank's z-slab
results of every operator along x, y and z, of the gradient and of the
laplacian must equal the single-field results bit for bit (the same lines go
through the same kernels; the z terms only travel through the transposes),
and match the oracle: max|x - r| / max|r| <= 1e-12."""
import numpy as np
import pytest

import oracle
from tests.fields import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("size", [2, 3, 4])
def test_slabs_equal_single_field(periodic, size):
    import torch

    import padeops_b200 as pb
    from padeops_b200 import _lib as L
    from padeops_b200 import field_ops as F
    from padeops_b200 import slabs as S

    shape = (96, 66, 64)  # n3, n2, n1: z and y not multiples of 4 or 3
    n3, n2, n1 = shape
    rng = np.random.default_rng(40 + size + periodic)
    f = rng.standard_normal(shape)
    g = torch.from_numpy(f).cuda()
    der = pb.Derivatives()
    dx = [2 * np.pi / n if periodic else 1.0 / (n - 1) for n in (n1, n2, n3)]
    der.init(n1, n2, n3, *dx, periodic, periodic, periodic, "cd10", "cd10", "cd10")
    whole = {}
    for axis in (1, 2, 3):
        for kind in (L.D1, L.D2):
            out = torch.empty_like(g)
            der.apply(kind, axis, g, out, 0, 0)
            whole[(axis, kind)] = out
    lap = torch.empty_like(g)
    F.laplacian(der, g, lap)
    torch.cuda.synchronize()
    for axis in (1, 2, 3):
        o = oracle.OracleOp(oracle.CD10, shape[3 - axis], dx[axis - 1], periodic)
        na, nb = {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]
        ref = o.apply(oracle.D1, axis, f, na, nb, 0, 0).reshape(shape)
        assert rel_err(whole[(axis, L.D1)].cpu().numpy(), ref) <= TOL, axis

    def rank(r, ex):
        s = S.Slabs(shape, size, r)
        fz = s.scatter(g)
        z0, z1 = s.z_range()
        for axis in (1, 2, 3):
            for kind in (L.D1, L.D2):
                d = torch.full_like(fz, float("nan"))
                S.apply(s, der.ops[axis - 1], kind, axis, fz, d, ex)
                assert torch.equal(d, whole[(axis, kind)][z0:z1]), (r, axis, kind)
        gx, gy, gz = (torch.full_like(fz, float("nan")) for _ in range(3))
        S.gradient(s, der, fz, gx, gy, gz, ex)
        for got, axis in ((gx, 1), (gy, 2), (gz, 3)):
            assert torch.equal(got, whole[(axis, L.D1)][z0:z1]), (r, axis)
        lz = torch.full_like(fz, float("nan"))
        S.laplacian(s, der, fz, lz, ex)
        assert torch.equal(lz, lap[z0:z1]), r
        torch.cuda.synchronize()
        return True

    assert all(S.run_local(size, rank))
