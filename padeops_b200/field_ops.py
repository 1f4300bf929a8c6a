"""Field operators built on the compact derivatives and filter: the single-GPU
counterparts of src/utilities/operators.F90 (gradient :18, curl :55,
divergence :118, filter3D :158).

The reference runs them on a 2DECOMP pencil decomposition, transposing between
x, y and z pencils for each direction.  Here the whole field is resident on
one GPU, so every direction is applied to the same (n3, n2, n1) array and no
transposes exist.  Boundary conventions are the reference's: each direction
takes a (bc1, bcn) pair, default (0, 0); divergence applies the negated pairs
(operators.F90:135-150); filter3D filters along y, then x, then z, each
`numtimes` times, and overwrites its input (operators.F90:180-222).

``der`` is a ``Derivatives`` and ``fil`` a ``Filters`` object
(padeops_b200.operators).  Fields are contiguous CUDA float64 tensors of shape
(n3, n2, n1).
"""
from __future__ import annotations

import torch

__all__ = ["gradient", "curl", "divergence", "filter3d"]

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
    (operators.F90:55-116); curlu has shape (3, n3, n2, n1)."""
    tmp = torch.empty_like(u)
    der.ddy(w, curlu[0], *y_bc)
    der.ddz(v, tmp, *z_bc)
    curlu[0].sub_(tmp)
    der.ddz(u, curlu[1], *z_bc)
    der.ddx(w, tmp, *x_bc)
    curlu[1].sub_(tmp)
    der.ddx(v, curlu[2], *x_bc)
    der.ddy(u, tmp, *y_bc)
    curlu[2].sub_(tmp)


def divergence(der, u: torch.Tensor, v: torch.Tensor, w: torch.Tensor, div: torch.Tensor,
               x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> None:
    """div = du/dx + dv/dy + dw/dz with the negated boundary pairs of the
    reference (operators.F90:118-156)."""
    tmp = torch.empty_like(u)
    der.ddy(v, div, -y_bc[0], -y_bc[1])
    der.ddx(u, tmp, -x_bc[0], -x_bc[1])
    div.add_(tmp)
    der.ddz(w, tmp, -z_bc[0], -z_bc[1])
    div.add_(tmp)


def filter3d(fil, arr: torch.Tensor, numtimes: int = 1, x_bc=_BC0, y_bc=_BC0, z_bc=_BC0) -> torch.Tensor:
    """Filters arr in place along y, then x, then z, numtimes times each
    (operators.F90:158-223); returns arr."""
    a, b = arr, torch.empty_like(arr)
    for filt, bc in ((fil.filtery, y_bc), (fil.filterx, x_bc), (fil.filterz, z_bc)):
        for _ in range(max(1, int(numtimes))):
            filt(a, b, *bc)
            a, b = b, a
    if a.data_ptr() != arr.data_ptr():
        arr.copy_(a)
    return arr
