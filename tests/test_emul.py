"""CPU emulation of the CUDA kernels: the device code of the line kernel and of
the streaming kernel (padeops_b200/csrc/*.cuh) compiled for the host, run
phase by phase over every thread of every CTA (tests/emul/pado_emul.cu), and
compared with the oracle.

This exercises the partition tables, the segment layouts, the coupling
windows, the constant-coefficient interior and the border responses without
a GPU; the GPU tests repeat the comparison on the device.  Tolerances:
forward <= 1e-12 relative to max |oracle|; the adjoint against the dense D^T
<= 1e-11 (the dense solve contributes its own rounding).
"""
import ctypes
import itertools

import numpy as np
import pytest

import oracle
from oracle import dense

OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]


@pytest.fixture(scope="module")
def emul():
    from tests.emul.build import build

    lib = ctypes.CDLL(build())
    P, I, D, Lg = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
    lib.emul_stream.argtypes = [I, I, I, D, I, I, I, I, I, I, P, P, Lg, Lg, I]
    lib.emul_apply.argtypes = [I, I, I, D, I, I, I, I, I, I, I, I, P, P, Lg, Lg, I]
    return lib


def _shape(n, axis):
    return {1: (3, 2, n), 2: (3, n, 5), 3: (n, 2, 9)}[axis]


def _bcs(scheme, periodic):
    return [(0, 0)] if periodic else [(0, 0), (1, -1), (-1, 1), (1, 1)]


def _rel(x, r):
    return float(np.abs(x - r).max() / np.abs(r).max())


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_stream_kernel_emulated(emul, scheme, kind, periodic):
    rng = np.random.default_rng(3 + scheme + 5 * kind)
    for n, m, lines in [(10, 32, 16), (34, 16, 8), (100, 32, 16), (256, 32, 16), (320, 64, 8), (512, 32, 16)]:
        for bc1, bcn in _bcs(scheme, periodic):
            dx = 0.37
            op = oracle.OracleOp(scheme, n, dx, periodic, bc1, bcn)
            for axis in (1, 2, 3):
                f = rng.standard_normal(_shape(n, axis))
                na, nb = [s for a, s in enumerate(f.shape[::-1]) if a != axis - 1]
                ref = op.apply(kind, axis, f, na, nb, bc1, bcn).reshape(f.shape)
                out = np.full_like(f, np.nan)
                rc = emul.emul_stream(scheme, kind, n, dx, int(periodic), bc1, bcn, m, lines, axis,
                                      f.ctypes.data, out.ctypes.data, na, nb, 0)
                assert rc == 0
                assert _rel(out, ref) <= 1e-12, (n, m, lines, bc1, bcn, axis, _rel(out, ref))


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_line_kernel_emulated(emul, scheme, kind, periodic):
    rng = np.random.default_rng(11 + scheme + 5 * kind)
    for n, m in [(13, 16), (64, 32), (100, 16)]:
        for bc1, bcn in _bcs(scheme, periodic):
            dx = 0.37
            op = oracle.OracleOp(scheme, n, dx, periodic, bc1, bcn)
            for axis, fast in itertools.product((1, 3), (1, 0)):
                f = rng.standard_normal(_shape(n, axis))
                na, nb = [s for a, s in enumerate(f.shape[::-1]) if a != axis - 1]
                ref = op.apply(kind, axis, f, na, nb, bc1, bcn).reshape(f.shape)
                out = np.full_like(f, np.nan)
                rc = emul.emul_apply(scheme, kind, n, dx, int(periodic), bc1, bcn, m, 4, 7, 0, axis,
                                     f.ctypes.data, out.ctypes.data, na, nb, fast)
                assert rc == 0
                assert _rel(out, ref) <= 1e-12, (n, m, bc1, bcn, axis, fast, _rel(out, ref))


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_adjoint_emulated(emul, scheme, kind, periodic):
    """The adjoint sweep (transformed tables, reversed recurrences) equals D^T."""
    rng = np.random.default_rng(17 + scheme + 5 * kind)
    for n, m in [(10, 16), (33, 16), (100, 32)]:
        for bc1, bcn in _bcs(scheme, periodic):
            dx = 0.37
            Dm = dense.operator(scheme, kind, n, dx, periodic, bc1, bcn)
            for axis, fast in itertools.product((1, 3), (1, 0)):
                g = rng.standard_normal(_shape(n, axis))
                na, nb = [s for a, s in enumerate(g.shape[::-1]) if a != axis - 1]
                ref = dense.apply_axis(Dm.T, g, axis)
                out = np.zeros_like(g)
                rc = emul.emul_apply(scheme, kind, n, dx, int(periodic), bc1, bcn, m, 4, 0, 1, axis,
                                     g.ctypes.data, out.ctypes.data, na, nb, fast)
                assert rc == 0
                assert _rel(out, ref) <= 1e-11, (n, m, bc1, bcn, axis, fast, _rel(out, ref))


@pytest.mark.parametrize("scheme,kind", OPS)
@pytest.mark.parametrize("periodic", [True, False])
def test_stream_adjoint_emulated(emul, scheme, kind, periodic):
    """The streaming kernel's adjoint (transposed sweep in the tile, then B^T)
    equals D^T from the dense assembly."""
    rng = np.random.default_rng(23 + scheme + 5 * kind)
    # (32, 32) and (64, 64): one segment, too few summary slots for the end
    # columns, so x lines store straight to global memory
    for n, m, lines in [(10, 32, 16), (32, 32, 16), (33, 16, 8), (64, 64, 8), (100, 32, 16), (256, 32, 16)]:
        for bc1, bcn in _bcs(scheme, periodic):
            dx = 0.37
            Dm = dense.operator(scheme, kind, n, dx, periodic, bc1, bcn)
            for axis in (1, 2, 3):
                g = rng.standard_normal(_shape(n, axis))
                na, nb = [s for a, s in enumerate(g.shape[::-1]) if a != axis - 1]
                ref = dense.apply_axis(Dm.T, g, axis)
                out = np.full_like(g, np.nan)
                rc = emul.emul_stream(scheme, kind, n, dx, int(periodic), bc1, bcn, m, lines, axis,
                                      g.ctypes.data, out.ctypes.data, na, nb, 1)
                assert rc == 0
                assert _rel(out, ref) <= 1e-11, (n, m, lines, bc1, bcn, axis, _rel(out, ref))
