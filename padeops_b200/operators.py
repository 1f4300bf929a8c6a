"""Reference-shaped scheme objects over the C ABI.

``cd06``, ``cd10`` and ``cf90`` mirror the Fortran types of
src/derivatives/cd06.F90, src/derivatives/cd10.F90 and src/filters/cf90.F90:
same method names (``init``, ``dd1``..``dd3``, ``d2d1``..``d2d3``,
``filter1``..``filter3``, ``destroy``, ``GetSize``), same argument order and
meaning, same ``ierr`` from ``init``.  ``Derivatives`` and ``Filters`` mirror
the serial ``DerivativesMod`` / ``FiltersMod`` dispatchers
(src/derivatives/derivatives.F90:140-187, 447-569; src/filters/filters.F90:
220-322) for the compact schemes.

Fields are CUDA float64 tensors holding the reference's column-major layout:
f(n1,n2,n3) is a tensor with n1*n2*n3 contiguous elements, f[i + n1*(j + n2*k)]
-- e.g. a C-contiguous torch tensor of shape (n3, n2, n1).  ``dd1(f, df, na,
nb)`` treats f as (n, na, nb), ``dd2`` as (na, n, nb), ``dd3`` as (na, nb, n),
exactly like the reference's explicit-shape dummies.  Work is enqueued on the
current torch CUDA stream.

Differences from the reference (by design): errors raise ``PadoError``
instead of aborting the MPI job (a bad bc raises with status 324, the code the
reference passes to GracefulExit), and every method also has an ``_adjoint``
form applying D^T.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import PadoError, check

__all__ = ["cd06", "cd10", "cf90", "Derivatives", "Filters", "PadoError"]


def _stream_ptr(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _check_field(t: torch.Tensor, numel: int, name: str) -> None:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (padeops_b200 has no CPU path)")
    if t.dtype != torch.float64:
        raise ValueError(f"{name} must be float64 (the reference computes in FP64)")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous (column-major field memory)")
    if t.numel() != numel:
        raise ValueError(f"{name} has {t.numel()} elements, expected {numel}")


class _Scheme:
    _scheme = -1

    def __init__(self):
        self._h = ctypes.c_void_p()
        self.n = 0
        self.periodic = True

    # -- life cycle ---------------------------------------------------------
    def _create(self, n: int, dx: float, periodic: bool, bc1: int, bcn: int) -> int:
        self.destroy()
        h = ctypes.c_void_p()
        ierr = L.lib().pado_create(ctypes.byref(h), self._scheme, int(n), float(dx), int(bool(periodic)),
                                   int(bc1), int(bcn))
        if ierr in (0,):
            self._h = h
            self.n = int(n)
            self.periodic = bool(periodic)
        elif ierr < 0:
            raise PadoError(ierr, f"{type(self).__name__}.init")
        return ierr

    def destroy(self) -> None:
        """%destroy (cd06.F90:203, cd10.F90:317, cf90.F90:177)."""
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().pado_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def GetSize(self) -> int:  # noqa: N802 (reference name)
        """%GetSize (cd06.F90:123, cd10.F90:189)."""
        return self.n

    @property
    def handle(self) -> int:
        if not self._h.value:
            raise PadoError(L.E_STATE, f"{type(self).__name__} used before a successful init")
        return self._h.value

    # -- tiling ---------------------------------------------------------------
    def set_tiling(self, m: int = 0, lines: int = 0) -> None:
        check(L.lib().pado_set_tiling(self.handle, m, lines), "set_tiling")

    def set_variant(self, variant: int) -> None:
        """0 = automatic, 1 = one CTA per tile of lines, 2/3 = persistent CTAs
        with prefetch, 4 = the streaming (TMA-fed) kernel, 5 = its resident
        tiles fed by plain loads, 6 = the streaming kernel fed by per-element
        asynchronous copies (5 and 6: any extent and 8-byte alignment)."""
        check(L.lib().pado_set_kernel_variant(self.handle, variant), "set_variant")

    def launch_plan(self, kind: int, axis: int, f: torch.Tensor, df: torch.Tensor, na: int, nb: int,
                    bc1: int = 0, bcn: int = 0) -> dict:
        """The kernel and tiling a forward apply with these arguments would use."""
        info = (ctypes.c_int * 8)()
        check(L.lib().pado_launch_plan(self.handle, kind, axis, ctypes.c_void_p(f.data_ptr()),
                                       ctypes.c_void_p(df.data_ptr()), na, nb, bc1, bcn, info), "launch_plan")
        keys = ("variant", "lines", "stages", "ctas_per_sm", "segments", "window", "threads", "smem")
        return dict(zip(keys, list(info)))

    def set_stream_tiling(self, lines: int = 0, stages: int = 0) -> None:
        """Lines per tile and shared-memory stages of the streaming kernel (0 = automatic)."""
        check(L.lib().pado_set_stream_tiling(self.handle, lines, stages), "set_stream_tiling")

    def device_status(self, clear: bool = True) -> int:
        """Status recorded by this handle's kernels (0, or PADO_E_TIMEOUT)."""
        rc = int(L.lib().pado_device_status(self.handle, 1 if clear else 0))
        if rc not in (L.OK, L.E_TIMEOUT):
            check(rc, "device_status")
        return rc

    def get_tiling(self) -> tuple[int, int]:
        m, lines = ctypes.c_int(), ctypes.c_int()
        check(L.lib().pado_get_tiling(self.handle, ctypes.byref(m), ctypes.byref(lines)), "get_tiling")
        return m.value, lines.value

    # -- generic apply ----------------------------------------------------------
    def apply(self, kind: int, axis: int, f: torch.Tensor, df: torch.Tensor, na: int, nb: int,
              bc1: int | None = None, bcn: int | None = None, adjoint: bool = False, alpha: float = 1.0,
              beta: float = 0.0) -> torch.Tensor:
        """df = alpha * D f + beta * df (beta 0 or 1; pado_apply_scaled), or
        D^T f for ``adjoint`` (alpha 1, beta 0 only)."""
        numel = self.n * int(na) * int(nb)
        _check_field(f, numel, "f")
        _check_field(df, numel, "df")
        if f.device != df.device:
            raise ValueError("f and df must be on the same device")
        b1, bn = 0 if bc1 is None else int(bc1), 0 if bcn is None else int(bcn)
        with torch.cuda.device(f.device):
            if alpha != 1.0 or beta != 0.0:
                if adjoint:
                    raise PadoError(L.E_UNSUPPORTED, "the adjoint has no scaled or accumulating form")
                st = L.lib().pado_apply_scaled(self.handle, kind, axis, f.data_ptr(), df.data_ptr(), int(na), int(nb),
                                               b1, bn, float(alpha), float(beta), _stream_ptr(f))
            else:
                fn = L.lib().pado_apply_adjoint if adjoint else L.lib().pado_apply
                st = fn(self.handle, kind, axis, f.data_ptr(), df.data_ptr(), int(na), int(nb), b1, bn, _stream_ptr(f))
        check(st, f"{type(self).__name__}.{'adjoint' if adjoint else 'apply'}(kind={kind}, axis={axis})")
        return df

    def apply_host(self, kind: int, axis: int, f, df, na: int, nb: int, bc1: int = 0, bcn: int = 0):
        """Host-buffer call (numpy arrays or CPU tensors, float64, contiguous): copies
        in, applies on the GPU, copies out; returns when df holds the result."""
        import numpy as np

        for name, a in (("f", f), ("df", df)):
            if isinstance(a, torch.Tensor):
                if a.is_cuda or a.dtype != torch.float64 or not a.is_contiguous():
                    raise ValueError(f"{name} must be a contiguous float64 host array")
            elif not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise ValueError(f"{name} must be a contiguous float64 host array")
        ptr = (lambda a: a.data_ptr() if isinstance(a, torch.Tensor) else a.ctypes.data)
        st = L.lib().pado_apply_host(self.handle, kind, axis, ptr(f), ptr(df), int(na), int(nb), int(bc1), int(bcn),
                                     torch.cuda.current_stream().cuda_stream)
        check(st, "apply_host")
        return df


class cd06(_Scheme):  # noqa: N801 (reference name)
    """6th-order compact first derivative (src/derivatives/cd06.F90)."""

    _scheme = L.CD06

    def init(self, n_: int, dx_: float, periodic_: bool, bc1_: int = 0, bcn_: int = 0) -> int:
        """cd06%init (cd06.F90:129): returns ierr (0; 3 periodic n in 2..5; 2 bounded n in 2..7)."""
        return self._create(n_, dx_, periodic_, bc1_, bcn_)

    def dd1(self, f, df, na, nb):
        """cd06%dd1 (cd06.F90:775): d/dx of f(n,na,nb)."""
        return self.apply(L.D1, 1, f, df, na, nb)

    def dd2(self, f, df, na, nb):
        """cd06%dd2 (cd06.F90:797): d/dy of f(na,n,nb)."""
        return self.apply(L.D1, 2, f, df, na, nb)

    def dd3(self, f, df, na, nb):
        """cd06%dd3 (cd06.F90:819): d/dz of f(na,nb,n)."""
        return self.apply(L.D1, 3, f, df, na, nb)

    def dd1_adjoint(self, g, fbar, na, nb):
        return self.apply(L.D1, 1, g, fbar, na, nb, adjoint=True)

    def dd2_adjoint(self, g, fbar, na, nb):
        return self.apply(L.D1, 2, g, fbar, na, nb, adjoint=True)

    def dd3_adjoint(self, g, fbar, na, nb):
        return self.apply(L.D1, 3, g, fbar, na, nb, adjoint=True)


class cd10(_Scheme):  # noqa: N801
    """10th-order compact first and second derivatives (src/derivatives/cd10.F90)."""

    _scheme = L.CD10

    def init(self, n_: int, dx_: float, periodic_: bool, bc1_: int = 0, bcn_: int = 0) -> int:
        """cd10%init (cd10.F90:195): returns ierr (0; 2 for n in 2..7)."""
        return self._create(n_, dx_, periodic_, bc1_, bcn_)

    def dd1(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cd10%dd1 (cd10.F90:2029)."""
        return self.apply(L.D1, 1, f, df, na, nb, bc1_, bcn_)

    def dd2(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cd10%dd2 (cd10.F90:2099)."""
        return self.apply(L.D1, 2, f, df, na, nb, bc1_, bcn_)

    def dd3(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cd10%dd3 (cd10.F90:2169)."""
        return self.apply(L.D1, 3, f, df, na, nb, bc1_, bcn_)

    def d2d1(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cd10%d2d1 (cd10.F90:2239)."""
        return self.apply(L.D2, 1, f, df, na, nb, bc1_, bcn_)

    def d2d2(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cd10%d2d2 (cd10.F90:2309)."""
        return self.apply(L.D2, 2, f, df, na, nb, bc1_, bcn_)

    def d2d3(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cd10%d2d3 (cd10.F90:2379)."""
        return self.apply(L.D2, 3, f, df, na, nb, bc1_, bcn_)


class cf90(_Scheme):  # noqa: N801
    """8th-order compact filter, 90% truncation (src/filters/cf90.F90)."""

    _scheme = L.CF90

    def init(self, n_: int, periodic_: bool) -> int:
        """cf90%init (cf90.F90:107): returns ierr (0; 7 for n in 2..9)."""
        return self._create(n_, 1.0, periodic_, 0, 0)

    def filter1(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cf90%filter1 (cf90.F90:1020)."""
        return self.apply(L.FILTER, 1, f, df, na, nb, bc1_, bcn_)

    def filter2(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cf90%filter2 (cf90.F90:1090)."""
        return self.apply(L.FILTER, 2, f, df, na, nb, bc1_, bcn_)

    def filter3(self, f, df, na, nb, bc1_=None, bcn_=None):
        """cf90%filter3 (cf90.F90:1160); a complex128 f and df take the complex
        variant (filter3_CMPLX, cf90.F90:1230-1251): right-hand side with the
        closures (bc1_, bcn_) -- bc1_ only when bcn_ is given, as in the
        reference -- and the solve with the bc (0,0) system."""
        if f.dtype == torch.complex128:
            if df.dtype != torch.complex128 or not (f.is_cuda and df.is_cuda and f.is_contiguous() and df.is_contiguous()):
                raise ValueError("complex filter3: f and df must be contiguous complex128 CUDA tensors")
            bc1, bcn = (0, 0) if bcn_ is None else (int(bc1_ or 0), int(bcn_))
            fr, dfr = torch.view_as_real(f), torch.view_as_real(df)
            with torch.cuda.device(f.device):
                st = L.lib().pado_filter3_complex(self.handle, fr.data_ptr(), dfr.data_ptr(), int(na), int(nb), bc1,
                                                  bcn, _stream_ptr(fr))
            check(st, "cf90.filter3 (complex)")
            return df
        return self.apply(L.FILTER, 3, f, df, na, nb, bc1_, bcn_)


_METHODS = {"cd10": (cd10, 1), "cd06": (cd06, 2)}


class Derivatives:
    """Serial ``DerivativesMod`` for the compact methods (derivatives.F90:140-187,
    276-389, 447-569).  Methods "four" and "cheb" are not part of this library."""

    def __init__(self):
        self.initialized = False

    def init(self, nx, ny, nz, dx, dy, dz, periodic_x, periodic_y, periodic_z, method_x, method_y, method_z):
        self.sz = (int(nx), int(ny), int(nz))
        self.ops = []
        for n, d, p, m in zip(self.sz, (dx, dy, dz), (periodic_x, periodic_y, periodic_z),
                              (method_x, method_y, method_z)):
            if m not in _METHODS:
                raise ValueError(f"derivative method {m!r} is not a compact scheme (cd10, cd06)")
            op = _METHODS[m][0]()
            ierr = op.init(n, d, p, 0, 0)
            if ierr != 0:
                raise PadoError(ierr, f"{m}.init(n={n})")
            self.ops.append(op)
        self.initialized = True
        return 0

    def _na_nb(self, axis):
        nx, ny, nz = self.sz
        return {1: (ny, nz), 2: (nx, nz), 3: (nx, ny)}[axis]

    def _d(self, kind, axis, f, df, bc1, bcn, alpha=1.0, beta=0.0):
        op = self.ops[axis - 1]
        if kind == L.D2 and isinstance(op, cd06):
            raise PadoError(L.E_UNSUPPORTED, "cd06 has no second derivative (derivatives.F90:525)")
        na, nb = self._na_nb(axis)
        if isinstance(op, cd06):
            bc1 = bcn = None
        elif bc1 is None or bcn is None:  # the bc pair is forwarded only when both are present
            bc1 = bcn = None
        return op.apply(kind, axis, f, df, na, nb, bc1, bcn, alpha=alpha, beta=beta)

    def apply(self, kind, axis, f, df, bc1=None, bcn=None, alpha=1.0, beta=0.0):
        """df = alpha * D f + beta * df along ``axis`` (1 x, 2 y, 3 z), D the first
        (kind 1) or second (kind 2) derivative of that direction's scheme."""
        return self._d(kind, axis, f, df, bc1, bcn, alpha, beta)

    def ddx(self, f, df, bc1=None, bcn=None):
        return self._d(L.D1, 1, f, df, bc1, bcn)

    def ddy(self, f, df, bc1=None, bcn=None):
        return self._d(L.D1, 2, f, df, bc1, bcn)

    def ddz(self, f, df, bc1=None, bcn=None):
        return self._d(L.D1, 3, f, df, bc1, bcn)

    def d2dx2(self, f, df, bc1=None, bcn=None):
        return self._d(L.D2, 1, f, df, bc1, bcn)

    def d2dy2(self, f, df, bc1=None, bcn=None):
        return self._d(L.D2, 2, f, df, bc1, bcn)

    def d2dz2(self, f, df, bc1=None, bcn=None):
        return self._d(L.D2, 3, f, df, bc1, bcn)

    def destroy(self):
        for op in getattr(self, "ops", []):
            op.destroy()
        self.initialized = False


class Filters:
    """Serial ``FiltersMod`` for the cf90 method (filters.F90:220-322)."""

    def init(self, nx, ny, nz, methodx, methody, methodz, periodicx, periodicy, periodicz):
        self.sz = (int(nx), int(ny), int(nz))
        self.ops = []
        for n, p, m in zip(self.sz, (periodicx, periodicy, periodicz), (methodx, methody, methodz)):
            if m != "cf90":
                raise ValueError(f"filter method {m!r} is not the compact filter (cf90)")
            op = cf90()
            ierr = op.init(n, p)
            if ierr != 0:
                raise PadoError(ierr, f"cf90.init(n={n})")
            self.ops.append(op)
        return 0

    def _f(self, axis, f, ff, bc1, bcn):
        nx, ny, nz = self.sz
        na, nb = {1: (ny, nz), 2: (nx, nz), 3: (nx, ny)}[axis]
        return self.ops[axis - 1].apply(L.FILTER, axis, f, ff, na, nb, bc1, bcn)

    def filterx(self, f, ff, bc1=None, bcn=None):
        return self._f(1, f, ff, bc1, bcn)

    def filtery(self, f, ff, bc1=None, bcn=None):
        return self._f(2, f, ff, bc1, bcn)

    def filterz(self, f, ff, bc1=None, bcn=None):
        return self._f(3, f, ff, bc1, bcn)

    def destroy(self):
        for op in getattr(self, "ops", []):
            op.destroy()
