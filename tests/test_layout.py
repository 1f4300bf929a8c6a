"""The segment layout every kernel sweeps (make_layout, pado_tables.cpp), for
every operator, boundary type, segment length and a range of line lengths
(odd ones and the configs' sizes included): the segments tile the line in
order, there are at most 32, and every constant-coefficient (fast) segment
has exactly m rows; at the configs' line lengths and default segment lengths
every other segment is one edge piece of exactly E rows, the fully unrolled
path's precondition (other lengths fall back to pieces of about m/3 rows on
the generic loop, which is correct but slower).  Host only."""
import ctypes

import numpy as np
import pytest

import oracle

OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]
LENGTHS = [8, 16, 31, 32, 33, 48, 63, 64, 65, 96, 100, 127, 128, 129, 192, 255, 256, 257, 384, 500, 511, 512,
           513, 640, 768, 1000, 1023, 1024]


@pytest.fixture(scope="module")
def emul():
    from tests.emul.build import build

    lib = ctypes.CDLL(build())
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.emul_layout.argtypes = [I, I, I, I, I, I, I, P, P, P, P, P]
    return lib


def _layout(lib, scheme, kind, n, periodic, m):
    starts = np.zeros(40, dtype=np.int32)
    fast = np.zeros(40, dtype=np.int32)
    S, E, W = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert lib.emul_layout(scheme, kind, n, int(periodic), 0, 0, m, starts.ctypes.data, fast.ctypes.data,
                           ctypes.byref(S), ctypes.byref(E), ctypes.byref(W)) == 0
    return starts[:S.value + 1], fast[:S.value], E.value, W.value


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("m", [16, 32, 64])
def test_layout_tiles_the_line(emul, scheme, kind, periodic, m):
    for n in LENGTHS:
        if (scheme == oracle.CF90 and n < 10) or n < 8 or (n + m - 1) // m > 32:
            continue  # below the scheme's minimum, or a segment length pado_set_tiling refuses
        starts, fast, E, W = _layout(emul, scheme, kind, n, periodic, m)
        lens = np.diff(starts)
        assert starts[0] == 0 and starts[-1] == n, (n, starts)
        assert (lens > 0).all(), (n, starts)
        assert len(lens) <= 32
        assert E >= 5 and W >= 0
        assert all(lens[s] == m for s in range(len(lens)) if fast[s]), (n, starts, fast)


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_default_tilings_use_whole_edge_pieces(emul, scheme, kind, periodic):
    """The configs' line lengths at the default segment length (32 rows below
    n = 1024, 64 from it): every segment outside the constant-coefficient
    block is an edge piece of exactly E rows (the unrolled path)."""
    for n in (128, 256, 384, 512, 640, 768, 1024):
        m = 64 if n >= 1024 else 32
        starts, fast, E, W = _layout(emul, scheme, kind, n, periodic, m)
        lens = np.diff(starts)
        if not fast.any():
            continue
        others = [int(lens[s]) for s in range(len(lens)) if not fast[s]]
        assert all(x == E for x in others), (n, m, E, starts)
