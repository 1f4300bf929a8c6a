"""CPU oracle for the compact-difference hot path (TEST INFRASTRUCTURE ONLY).

This package is the parity checker for ``padeops_b200``: a C restatement
(``pado_oracle.c``) of the reference Fortran modules ``cd06stuff``
(src/derivatives/cd06.F90), ``cd10stuff`` (src/derivatives/cd10.F90) and
``cf90stuff`` (src/filters/cf90.F90), plus ``dense.py``, an independent dense
assembly of the same operators used to cross-check the restatement and to
build D^T for the adjoint checks.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs import it.  The product (``padeops_b200``) never does.

How it is pinned: the reference cannot be built here (it is Fortran and no
Fortran compiler exists on either machine), so the restatement is checked
against the reference's own closed-form known answers -- the modified
wavenumbers / transfer function of ``src/utilities/spectral.F90:938-1010`` for
periodic Fourier modes, which the discrete operators reproduce to rounding --
against the reference tests' recipes (``tests/test_cd06.F90``,
``test_cd10.F90``, ``test_cd10_NP.F90``, ``test_cd10_der2.F90``,
``test_cf90.F90``), and against ``dense.py``.  See tests/test_oracle.py.

Array convention (same as the reference): a field f(n1,n2,n3) is stored
column-major, f[i + n1*(j + n2*k)].  In numpy that is a C-ordered array of
shape (n3, n2, n1).  ``apply`` takes any contiguous float64 array with
n*na*nb elements and interprets it as the reference's explicit-shape dummy
(n,na,nb) / (na,n,nb) / (na,nb,n) for axis 1 / 2 / 3.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

__all__ = ["OracleOp", "build", "library", "CD06", "CD10", "CF90", "D1", "D2", "FILTER"]

CD06, CD10, CF90 = 0, 1, 2
FILTER, D1, D2 = 0, 1, 2

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_libs: dict[str, ctypes.CDLL] = {}


def build() -> None:
    """Compile the oracle libraries (make in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def library(fast: bool = False) -> ctypes.CDLL:
    """Load (building on demand) the strict or the fast-flags oracle library."""
    name = "libpado_oracle_fast.so" if fast else "libpado_oracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(_BUILD, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    lib.oracle_create.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.oracle_create.restype = ctypes.c_int
    lib.oracle_destroy.argtypes = [P]
    lib.oracle_destroy.restype = None
    lib.oracle_apply.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_long, ctypes.c_long,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.oracle_apply.restype = ctypes.c_int
    lib.oracle_table.argtypes = [P, ctypes.c_int, P]
    lib.oracle_table.restype = ctypes.c_int
    lib.oracle_filter3_complex.argtypes = [P, P, P, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int]
    lib.oracle_filter3_complex.restype = ctypes.c_int
    _libs[name] = lib
    return lib


class OracleOp:
    """One reference scheme object: cd06/cd10 ``init(n, dx, periodic, bc1, bcn)``
    (cd06.F90:129, cd10.F90:195) or cf90 ``init(n, periodic)`` (cf90.F90:107).

    ``ierr`` holds the reference's init status (0, or 3/2 for cd06, 2 for
    cd10, 7 for cf90 when n is too small).
    """

    def __init__(self, scheme: int, n: int, dx: float = 1.0, periodic: bool = True,
                 bc1: int = 0, bcn: int = 0, fast: bool = False):
        self.lib = library(fast)
        self.scheme, self.n, self.dx, self.periodic = scheme, n, dx, periodic
        self.bc1, self.bcn = bc1, bcn
        h = ctypes.c_void_p()
        self.ierr = self.lib.oracle_create(ctypes.byref(h), scheme, n, float(dx), int(bool(periodic)), bc1, bcn)
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self.lib.oracle_destroy(h)
            self._h = None

    def apply(self, kind: int, axis: int, f: np.ndarray, na: int, nb: int, bc1: int = 0, bcn: int = 0,
              nthreads: int = 1, out: np.ndarray | None = None) -> np.ndarray:
        """dd{axis} (kind=D1), d2d{axis} (kind=D2) or filter{axis} (kind=FILTER)."""
        if self.ierr != 0:
            raise RuntimeError(f"oracle operator failed init with ierr={self.ierr}")
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.size != self.n * na * nb:
            raise ValueError(f"field has {f.size} elements, expected {self.n * na * nb}")
        df = np.empty_like(f) if out is None else out
        rc = self.lib.oracle_apply(self._h, kind, axis, f.ctypes.data, df.ctypes.data, na, nb, bc1, bcn, nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle_apply returned {rc}")
        return df

    def filter3_complex(self, f: np.ndarray, na: int, nb: int, bc1: int = 0, bcn: int = 0,
                        nthreads: int = 1) -> np.ndarray:
        """cf90%filter3 of a complex (na,nb,n) field (filter3_CMPLX, cf90.F90:1230):
        right-hand side with closures (bc1, bcn), solve with the bc (0,0) system."""
        f = np.ascontiguousarray(f, dtype=np.complex128)
        if f.size != self.n * na * nb:
            raise ValueError(f"field has {f.size} elements, expected {self.n * na * nb}")
        df = np.empty_like(f)
        rc = self.lib.oracle_filter3_complex(self._h, f.ctypes.data, df.ctypes.data, na, nb, bc1, bcn, nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle_filter3_complex returned {rc}")
        return df

    def table(self, which: int, ncol: int) -> np.ndarray:
        """Coefficient table (n, ncol) as the reference stores it (column-major)."""
        buf = np.zeros(self.n * ncol, dtype=np.float64)
        if self.lib.oracle_table(self._h, which, buf.ctypes.data) != 0:
            raise ValueError("no such table")
        return buf.reshape(ncol, self.n).T.copy()
