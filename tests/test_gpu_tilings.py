"""GPU: every tiling of the streaming kernel the planner can choose -- 8, 16
and 32 lines per tile, one or two shared-memory stages, tensor / bulk copies
(variant 4) and per-element copies (variant 6) -- along every axis, periodic
and bounded, against the oracle (max|x - r| / max|r| <= 1e-12).  A tiling
that does not fit a line length is refused (PADO_E_UNSUPPORTED under variants
4 and 6), which the test accepts; each case checks that at least one tiling
ran."""
import numpy as np
import pytest

import oracle
from tests.fields import na_nb, rel_err
from tests.test_gpu_parity import OPS, _make, _oracle_apply

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("n", [96, 256])
def test_every_stream_tiling(scheme, kind, n):
    import torch

    from padeops_b200 import _lib as L

    rng = np.random.default_rng(90 + n + 5 * scheme + kind)
    shapes = {1: (6, 70, n), 2: (5, n, 66), 3: (n, 5, 66)}
    for periodic in (True, False):
        op = _make(scheme, n, 0.3, periodic)
        for axis in (1, 2, 3):
            shape = shapes[axis]
            f = rng.standard_normal(shape)
            ft = torch.from_numpy(f).cuda()
            na, nb = na_nb(shape, axis)
            bc = (0, 0) if periodic or scheme == oracle.CD06 else (1, -1)
            ref = _oracle_apply(scheme, kind, axis, f, 0.3, periodic, *bc)
            ran = 0
            for variant in (4, 6):
                op.set_variant(variant)
                for lines in (8, 16, 32):
                    for stages in (1, 2):
                        op.set_stream_tiling(lines, stages)
                        out = torch.full_like(ft, float("nan"))
                        try:
                            op.apply(kind, axis, ft, out, na, nb, *bc)
                        except L.PadoError as e:
                            assert e.status == L.E_UNSUPPORTED, e
                            continue
                        torch.cuda.synchronize()
                        plan = op.launch_plan(kind, axis, ft, out, na, nb, *bc)
                        assert (plan["variant"], plan["lines"], plan["stages"]) == (variant, lines, stages), plan
                        assert op.device_status() == 0
                        err = rel_err(out.cpu().numpy(), ref)
                        assert err <= TOL, (periodic, axis, variant, lines, stages, err)
                        ran += 1
            op.set_stream_tiling(0, 0)
            op.set_variant(0)
            assert ran > 0, (periodic, axis)
