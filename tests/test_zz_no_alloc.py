"""GPU: pado_batch_run_static, the batched launch that allocates no device
memory (for solvers that hand all of HBM to their own pool at start-up, or
that build a new list of fields every step and may not cudaMalloc while they
run).  Its descriptors and tile counter sit in one fixed array inside the
library, shared by every call.

Checked through the C ABI against pado_apply, item by item, on two calls in
a row with different item lists (so the second call meets the first call's
leftovers in the shared array), with the tolerance of the other parity
tests: max|x - r| / max|r| <= 1e-12.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _workload(torch, nitems, seed):
    import padeops_b200 as pb
    from padeops_b200._lib import CD06, CD10, CF90, D1, D2, FILTER

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nitems):
        shape = tuple(int(v) for v in rng.choice((32, 48, 64, 96), size=3))
        scheme = int(rng.choice([CD06, CD10, CF90]))
        kind = {CD06: D1, CF90: FILTER}.get(scheme, int(rng.choice([D1, D2])))
        periodic = bool(rng.integers(2))
        axis = int(rng.integers(1, 4))
        n = shape[3 - axis]
        bc1, bcn = (0, 0) if periodic else (int(rng.choice([0, 1, -1])), int(rng.choice([0, 1, -1])))
        op = {CD06: pb.cd06, CD10: pb.cd10, CF90: pb.cf90}[scheme]()
        ibc = (bc1, bcn) if scheme == CD06 else (0, 0)
        ierr = op.init(n, periodic) if scheme == CF90 else op.init(n, 0.3, periodic, *ibc)
        assert ierr == 0
        f = torch.from_numpy(rng.standard_normal(shape)).cuda()
        out.append((op, kind, axis, f, torch.full_like(f, float("nan")), bc1, bcn))
    return out


def _run_static(torch, items):
    from padeops_b200 import _lib as L

    arr = (L.BatchItem * len(items))()
    for i, (op, kind, axis, f, df, bc1, bcn) in enumerate(items):
        n3, n2, n1 = f.shape
        arr[i] = L.BatchItem(op.handle, kind, axis, bc1, bcn, n1, n2, n3, f.data_ptr(), df.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    return L.lib().pado_batch_run_static(ctypes.cast(arr, ctypes.c_void_p), len(items), stream)


def _check_against_apply(torch, items):
    torch.cuda.synchronize()
    for op, kind, axis, f, df, bc1, bcn in items:
        n3, n2, n1 = f.shape
        na, nb = {1: (n2, n3), 2: (n1, n3), 3: (n1, n2)}[axis]
        ref = torch.empty_like(f)
        op.apply(kind, axis, f, ref, na, nb, bc1, bcn)
        torch.cuda.synchronize()
        err = (df - ref).abs().max().item() / ref.abs().max().item()
        assert err <= TOL, (kind, axis, tuple(f.shape), err)


def test_static_batch_matches_apply_on_two_calls():
    import torch

    first = _workload(torch, 40, seed=1)
    second = _workload(torch, 23, seed=2)
    assert _run_static(torch, first) == 0
    _check_against_apply(torch, first)
    assert _run_static(torch, second) == 0
    _check_against_apply(torch, second)


def test_static_batch_allocates_nothing_and_calls_back_to_back():
    """Two calls in a row on one stream with no synchronization between them
    (the second call's descriptor copies wait behind the first launch on the
    stream), then both outputs against pado_apply; device memory in use --
    the driver's count and torch's -- is the same before and after."""
    import torch

    first = _workload(torch, 31, seed=4)
    second = _workload(torch, 17, seed=5)
    assert _run_static(torch, first) == 0  # the first call on this device sets up the scratch address
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for it in first + second:
        it[4].fill_(float("nan"))
    torch.cuda.synchronize()
    assert _run_static(torch, first) == 0
    assert _run_static(torch, second) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert free1 == free0
    _check_against_apply(torch, first)
    _check_against_apply(torch, second)


def test_static_batch_rejects_too_many_items():
    import torch

    from padeops_b200 import _lib as L

    items = _workload(torch, 1, seed=3) * (L.STATIC_BATCH_MAX_ITEMS + 1)
    assert _run_static(torch, items) == L.E_SIZE
