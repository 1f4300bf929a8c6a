"""Batched execution: many (field, operator) items in one persistent launch.

``Batch`` wraps pado_batch_create / pado_batch_run / pado_batch_run_graph /
pado_batch_run_loop.  Every item names a scheme object (cd06 / cd10 / cf90),
the operator kind and axis, the closures, and a field of shape (n3, n2, n1)
(CUDA float64, contiguous) with its output.  Tensors are kept alive by the
batch object.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import check

__all__ = ["Batch"]


class Batch:
    def __init__(self, items):
        """items: iterable of (op, kind, axis, f, df, bc1, bcn); f/df CUDA
        float64 tensors of shape (n3, n2, n1)."""
        self._keep = []
        arr = (L.BatchItem * max(1, len(items)))()
        for i, (op, kind, axis, f, df, bc1, bcn) in enumerate(items):
            if f.dim() != 3 or f.shape != df.shape or not (f.is_cuda and df.is_cuda):
                raise ValueError("batch fields must be 3-d CUDA tensors of equal shape (n3, n2, n1)")
            if f.dtype != torch.float64 or df.dtype != torch.float64 or not f.is_contiguous() or not df.is_contiguous():
                raise ValueError("batch fields must be contiguous float64")
            n3, n2, n1 = f.shape
            arr[i] = L.BatchItem(op.handle, kind, axis, bc1, bcn, n1, n2, n3, f.data_ptr(), df.data_ptr())
            self._keep.append((op, f, df))
        self._h = ctypes.c_void_p()
        check(L.lib().pado_batch_create(ctypes.byref(self._h), arr, len(items)), "pado_batch_create")

    def _stream(self) -> int:
        return torch.cuda.current_stream().cuda_stream

    def run(self) -> None:
        """One persistent launch over all items."""
        check(L.lib().pado_batch_run(self._h, self._stream()), "pado_batch_run")

    def run_graph(self) -> None:
        """Replay the persistent launch from a CUDA graph (captured on first use)."""
        check(L.lib().pado_batch_run_graph(self._h, self._stream()), "pado_batch_run_graph")

    def run_loop(self) -> None:
        """One launch per item (the per-field loop the batch replaces)."""
        check(L.lib().pado_batch_run_loop(self._h, self._stream()), "pado_batch_run_loop")

    def set_graph_branches(self, branches: int) -> int:
        """What run_graph captures: 0 = the persistent launch, k > 0 = one
        streaming-kernel launch per item on k concurrent graph branches."""
        return L.lib().pado_batch_set_graph_branches(self._h, branches)

    def set_config(self, lines: int = 0, ctas_per_sm: int = 0) -> int:
        """Lines per tile (8, 16, 32, 64; 0 = automatic) and a cap on CTAs per SM (0 = none)."""
        return L.lib().pado_batch_set_config(self._h, lines, ctas_per_sm)

    def status(self) -> int:
        """Device status of the last persistent launch: 0, or E_TIMEOUT when a
        CTA's bounded wait for its tile copies expired (synchronous)."""
        return L.lib().pado_batch_status(self._h)

    def info(self) -> dict:
        nt, grid, thr, smem = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        check(L.lib().pado_batch_info(self._h, ctypes.byref(nt), ctypes.byref(grid), ctypes.byref(thr),
                                      ctypes.byref(smem)), "pado_batch_info")
        return {"tiles": nt.value, "grid": grid.value, "threads": thr.value, "smem_bytes": smem.value}

    def destroy(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().pado_batch_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
