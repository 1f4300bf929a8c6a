"""The staggered sixth-order compact scheme over the C ABI, shaped like the
reference type ``cd06stagg`` (src/derivatives/cd06stagg.F90): ``init`` (the
periodic form ``init(nx, dx)`` or the non-periodic one with the boundary
types), ``ddz_E2C``, ``ddz_C2E``, ``ddz_C2C``, ``ddz_E2E``, ``d2dz2_C2C``,
``d2dz2_E2E``, ``InterpZ_E2C``, ``InterpZ_C2E`` and ``destroy``.

Fields are CUDA tensors holding the reference's column-major (n1, n2, nz)
arrays -- C-contiguous (nz, n2, n1) tensors -- float64, or complex128 (the
real and imaginary parts are processed as interleaved doubles).  Edge fields
have n + 1 planes, cell fields n.  Work is enqueued on the current stream.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import PadoError, check

__all__ = ["cd06stagg"]

_OPS = {"ddz_E2C": 0, "ddz_C2E": 1, "ddz_C2C": 2, "ddz_E2E": 3, "d2dz2_C2C": 4, "d2dz2_E2E": 5,
        "InterpZ_E2C": 6, "InterpZ_C2E": 7}


class cd06stagg:  # noqa: N801 (reference name)
    def __init__(self):
        self._h = ctypes.c_void_p()
        self.n = 0

    def init(self, nx: int, dx: float, isTopEven: bool | None = None, isBotEven: bool | None = None,  # noqa: N803
             isTopSided: bool = False, isBotSided: bool = False) -> int:  # noqa: N803
        """init_periodic(nx, dx) when no boundary types are given, else
        init_nonperiodic(nx, dx, isTopEven, isBotEven, isTopSided, isBotSided)
        (cd06stagg.F90:170, 197).  Returns 0, or PADO_STAGG_E_SHORT (21) for
        nx <= 4 (the reference's exit code)."""
        self.destroy()
        h = ctypes.c_void_p()
        if isTopEven is None and isBotEven is None:
            rc = L.lib().pado_cd06stagg_init_periodic(ctypes.byref(h), int(nx), float(dx))
        else:
            rc = L.lib().pado_cd06stagg_init_nonperiodic(ctypes.byref(h), int(nx), float(dx), int(bool(isTopEven)),
                                                         int(bool(isBotEven)), int(bool(isTopSided)),
                                                         int(bool(isBotSided)))
        if rc == 0:
            self._h = h
            self.n = int(nx)
        elif rc < 0:
            raise PadoError(rc, "cd06stagg.init")
        return rc

    def destroy(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().pado_cd06stagg_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def sizes(self, name: str) -> tuple[int, int]:
        """(planes read, planes written) of an operator: n or n + 1."""
        nin, nout = ctypes.c_int(), ctypes.c_int()
        check(L.lib().pado_cd06stagg_sizes(self._handle(), _OPS[name], ctypes.byref(nin), ctypes.byref(nout)), name)
        return nin.value, nout.value

    def _handle(self) -> int:
        if not self._h.value:
            raise PadoError(L.E_STATE, "cd06stagg used before a successful init")
        return self._h.value

    def _apply(self, name: str, f: torch.Tensor, df: torch.Tensor, n1: int, n2: int) -> torch.Tensor:
        nin, nout = self.sizes(name)
        cplx = f.is_complex()
        for t, nm, planes in ((f, "f", nin), (df, "df", nout)):
            if not isinstance(t, torch.Tensor) or not t.is_cuda:
                raise ValueError(f"{nm} must be a CUDA tensor (padeops_b200 has no CPU path)")
            if t.dtype != (torch.complex128 if cplx else torch.float64) or not t.is_contiguous():
                raise ValueError(f"{nm} must be a contiguous float64 or complex128 tensor, like f")
            if t.numel() != int(n1) * int(n2) * planes:
                raise ValueError(f"{nm} has {t.numel()} elements, expected {n1}*{n2}*{planes}")
        m1 = 2 * int(n1) if cplx else int(n1)
        with torch.cuda.device(f.device):
            st = L.lib().pado_cd06stagg_apply(self._handle(), _OPS[name], f.data_ptr(), df.data_ptr(), m1, int(n2),
                                              torch.cuda.current_stream(f.device).cuda_stream)
        check(st, f"cd06stagg.{name}")
        return df

    def ddz_E2C(self, fE, dfC, n1, n2):  # noqa: N802 (reference names below)
        """cd06stagg.F90:820"""
        return self._apply("ddz_E2C", fE, dfC, n1, n2)

    def ddz_C2E(self, fC, dfE, n1, n2):  # noqa: N802
        """cd06stagg.F90:850"""
        return self._apply("ddz_C2E", fC, dfE, n1, n2)

    def ddz_C2C(self, fC, dfC, n1, n2):  # noqa: N802
        """cd06stagg.F90:883"""
        return self._apply("ddz_C2C", fC, dfC, n1, n2)

    def ddz_E2E(self, fE, dfE, n1, n2):  # noqa: N802
        """cd06stagg.F90:905"""
        return self._apply("ddz_E2E", fE, dfE, n1, n2)

    def d2dz2_C2C(self, fC, d2fC, n1, n2):  # noqa: N802
        """cd06stagg.F90:995"""
        return self._apply("d2dz2_C2C", fC, d2fC, n1, n2)

    def d2dz2_E2E(self, fE, d2fE, n1, n2):  # noqa: N802
        """cd06stagg.F90:1027"""
        return self._apply("d2dz2_E2E", fE, d2fE, n1, n2)

    def InterpZ_E2C(self, fE, IfC, n1, n2):  # noqa: N802
        """cd06stagg.F90:928"""
        return self._apply("InterpZ_E2C", fE, IfC, n1, n2)

    def InterpZ_C2E(self, fC, IfE, n1, n2):  # noqa: N802
        """cd06stagg.F90:960"""
        return self._apply("InterpZ_C2E", fC, IfE, n1, n2)
