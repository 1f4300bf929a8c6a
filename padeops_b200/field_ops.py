"""Field operators built on the compact derivatives and filter: the single-GPU
counterparts of src/utilities/operators.F90 (gradient :18, curl :55,
divergence :118, filter3D :158) and of cgrid%laplacian
(src/compressible/cgrid.F90:480-517).

The reference runs them on a 2DECOMP pencil decomposition, transposing between
x, y and z pencils for each direction and summing the terms of a curl,
divergence or laplacian through pencil temporaries.  Here the whole field is
resident on one GPU, so every direction is applied to the same (n3, n2, n1)
array, and each sum is formed inside the operators' kernels: the first term
is stored, every further term is added into the output by the accumulating
form of the apply (pado_apply_scaled, beta = 1), so no temporary field and no
separate elementwise pass exist.  The terms are summed in the reference's
order and each addition rounds once, as the reference's `a = a + b` does.

Boundary conventions are the reference's: each direction takes a (bc1, bcn)
pair, default (0, 0); divergence applies the negated pairs
(operators.F90:135-150); filter3D filters along y, then x, then z, each
`numtimes` times, and overwrites its input (operators.F90:180-222).

``der`` is a ``Derivatives`` and ``fil`` a ``Filters`` object
(padeops_b200.operators).  Fields are contiguous CUDA float64 tensors of shape
(n3, n2, n1).
"""
from __future__ import annotations

import torch

from . import _lib as L

__all__ = ["gradient", "curl", "divergence", "laplacian", "filter3d", "apply_host_terms", "gradient_host",
           "laplacian_host"]

_BC0 = (0, 0)


def gradient(der, f: torch.Tensor, dfdx: torch.Tensor, dfdy: torch.Tensor, dfdz: torch.Tensor,
             x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """dfdx, dfdy, dfdz = the x, y, z first derivatives of f (operators.F90:18-53)."""
    der.ddy(f, dfdy, *y_bc)
    der.ddx(f, dfdx, *x_bc)
    der.ddz(f, dfdz, *z_bc)


def curl(der, u: torch.Tensor, v: torch.Tensor, w: torch.Tensor, curlu: torch.Tensor,
         x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """curlu[0] = dw/dy - dv/dz, curlu[1] = du/dz - dw/dx, curlu[2] = dv/dx - du/dy
    (operators.F90:55-116); curlu has shape (3, n3, n2, n1).  The subtracted
    derivative is accumulated with alpha = -1."""
    der.apply(L.D1, 2, w, curlu[0], *y_bc)
    der.apply(L.D1, 3, v, curlu[0], *z_bc, alpha=-1.0, beta=1.0)
    der.apply(L.D1, 3, u, curlu[1], *z_bc)
    der.apply(L.D1, 1, w, curlu[1], *x_bc, alpha=-1.0, beta=1.0)
    der.apply(L.D1, 1, v, curlu[2], *x_bc)
    der.apply(L.D1, 2, u, curlu[2], *y_bc, alpha=-1.0, beta=1.0)


def divergence(der, u: torch.Tensor, v: torch.Tensor, w: torch.Tensor, div: torch.Tensor,
               x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """div = dv/dy + du/dx + dw/dz, summed in that order, with the negated
    boundary pairs of the reference (operators.F90:118-156)."""
    der.apply(L.D1, 2, v, div, -y_bc[0], -y_bc[1])
    der.apply(L.D1, 1, u, div, -x_bc[0], -x_bc[1], beta=1.0)
    der.apply(L.D1, 3, w, div, -z_bc[0], -z_bc[1], beta=1.0)


def laplacian(der, f: torch.Tensor, lapf: torch.Tensor, x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """lapf = d2f/dy2 + d2f/dx2 + d2f/dz2, summed in that order
    (cgrid.F90:480-517); every direction needs a cd10 derivative (cd06 has no
    second derivative, derivatives.F90:525)."""
    der.apply(L.D2, 2, f, lapf, *y_bc)
    der.apply(L.D2, 1, f, lapf, *x_bc, beta=1.0)
    der.apply(L.D2, 3, f, lapf, *z_bc, beta=1.0)


def filter3d(fil, arr: torch.Tensor, numtimes: int = 1, x_bc=_BC0, y_bc=_BC0, z_bc=_BC0,
             work: torch.Tensor | None = None) -> torch.Tensor:
    """Filters arr in place along y, then x, then z, numtimes times each
    (operators.F90:158-223); returns arr.  A filter cannot overwrite its own
    input, so the passes alternate between arr and one work field of the same
    shape (``work``, allocated when not given; the reference uses pencil
    temporaries the same way)."""
    b = torch.empty_like(arr) if work is None else work
    a = arr
    for filt, bc in ((fil.filtery, y_bc), (fil.filterx, x_bc), (fil.filterz, z_bc)):
        for _ in range(max(1, int(numtimes))):
            filt(a, b, *bc)
            a, b = b, a
    if a.data_ptr() != arr.data_ptr():
        arr.copy_(a)
    return arr


def _host_ptr(a) -> int:
    import numpy as np

    if isinstance(a, torch.Tensor):
        if a.is_cuda or a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("host fields must be contiguous float64 CPU arrays")
        return a.data_ptr()
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
        raise ValueError("host fields must be contiguous float64 CPU arrays")
    return a.ctypes.data


def apply_host_terms(f, shape, terms, outs) -> None:
    """Host-buffer field operator (pado_apply_host_terms): f uploaded once, then
    every term (op, kind, axis, bc1, bcn, alpha, beta, out) applied into
    outs[out] on the device; each output is copied back while the next is
    computed.  shape = (n3, n2, n1) of the column-major field."""
    import ctypes

    n3, n2, n1 = (int(v) for v in shape)
    arr = (L.HostTerm * len(terms))()
    for i, (op, kind, axis, bc1, bcn, alpha, beta, out) in enumerate(terms):
        arr[i] = L.HostTerm(op.handle, kind, axis, bc1, bcn, alpha, beta, out)
    ptrs = (ctypes.c_void_p * len(outs))(*[_host_ptr(o) for o in outs])
    st = L.lib().pado_apply_host_terms(_host_ptr(f), n1, n2, n3, arr, len(terms), ptrs, len(outs),
                                      torch.cuda.current_stream().cuda_stream)
    L.check(st, "apply_host_terms")


def gradient_host(der, f, dfdx, dfdy, dfdz, x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """gradient of a host field: one upload, three results copied back."""
    ops = der.ops
    apply_host_terms(f, f.shape, [(ops[1], L.D1, 2, *y_bc, 1.0, 0.0, 0), (ops[0], L.D1, 1, *x_bc, 1.0, 0.0, 1),
                                  (ops[2], L.D1, 3, *z_bc, 1.0, 0.0, 2)], [dfdy, dfdx, dfdz])


def laplacian_host(der, f, lapf, x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """laplacian of a host field: one upload, the three terms summed on the
    device, one result copied back."""
    ops = der.ops
    apply_host_terms(f, f.shape, [(ops[1], L.D2, 2, *y_bc, 1.0, 0.0, 0), (ops[0], L.D2, 1, *x_bc, 1.0, 1.0, 0),
                                  (ops[2], L.D2, 3, *z_bc, 1.0, 1.0, 0)], [lapf])
