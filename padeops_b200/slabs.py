"""Distributed-field mode: one (n3, n2, n1) field larger than one GPU, split
over the ranks of a process group in z-slabs, with the compact operators
applied along every axis.

The reference keeps its fields in 2DECOMP pencils and moves them between
pencil orientations with ALLTOALLV transposes around every derivative across
the distributed direction (src/utilities/operators.F90:40-51: transpose_y_to_x
before ddx, transpose_y_to_z before ddz, and back).  Here each rank holds a
z-slab -- planes z0..z1-1, all of x and y -- so x and y lines are whole on
every rank and their derivatives, filters and accumulations run locally with
no communication.  Only the z direction moves data: one all-to-all takes the
z-slabs to y-slabs (every rank then holds all z for a range of y, so z lines
are whole), the operator runs there, and one all-to-all brings the result
back.  With 180 GB of HBM per GPU a slab of a 2048^3 FP64 field fits on 8
ranks, so a one-dimensional split is enough; the exchanges are NCCL
all-to-all over NVLink / NVSwitch (torch.distributed, any backend that has
all_to_all_single: nccl on GPUs, gloo on the host for tests).

Data movement per z operator: every rank sends (P - 1) / P of its slab and
receives as much, twice (there and back).  Packing is one contiguous copy on
the way out (y chunks of the z-slab); the y-slab arrives already in z order,
and the way back lands in z order and is unpacked by one copy.

The exchange is a callable (send, send_counts, recv_counts) -> received, so
that the same code runs with NCCL, gloo, or an in-process emulation of the
ranks in host threads (``LocalExchange``, ``run_local``), which the tests use
to check the packing on one GPU and the ranks' agreement on the host.
"""
from __future__ import annotations

from typing import Callable, Sequence

import torch

from . import _lib as L

__all__ = ["Slabs", "dist_exchange", "LocalExchange", "run_local", "transpose_z_to_y", "transpose_y_to_z", "apply",
           "gradient", "laplacian"]

Exchange = Callable[[torch.Tensor, Sequence[int], Sequence[int]], torch.Tensor]


def _split(n: int, parts: int, i: int) -> tuple[int, int]:
    """[lo, hi) of part i when n items are dealt to `parts` parts, the first
    n % parts parts taking one more."""
    q, r = divmod(n, parts)
    lo = i * q + min(i, r)
    return lo, lo + q + (1 if i < r else 0)


class Slabs:
    """The z-slab / y-slab decomposition of an (n3, n2, n1) field over
    `size` ranks; this rank is `rank`.

    z-slab of rank r: planes z_range(r), shape (nz_r, n2, n1), the resident
    layout.  y-slab of rank r: rows y_range(r) of every plane, shape
    (n3, ny_r, n1), the layout z operators run in.
    """

    def __init__(self, shape: Sequence[int], size: int, rank: int):
        n3, n2, n1 = (int(v) for v in shape)
        if size < 1 or not 0 <= rank < size:
            raise ValueError("rank must lie in [0, size)")
        if min(n3, n2, n1) < 1:
            raise ValueError("every extent must be positive")
        self.shape = (n3, n2, n1)
        self.size = size
        self.rank = rank

    def z_range(self, r: int | None = None) -> tuple[int, int]:
        return _split(self.shape[0], self.size, self.rank if r is None else r)

    def y_range(self, r: int | None = None) -> tuple[int, int]:
        return _split(self.shape[1], self.size, self.rank if r is None else r)

    def z_shape(self, r: int | None = None) -> tuple[int, int, int]:
        z0, z1 = self.z_range(r)
        return (z1 - z0, self.shape[1], self.shape[2])

    def y_shape(self, r: int | None = None) -> tuple[int, int, int]:
        y0, y1 = self.y_range(r)
        return (self.shape[0], y1 - y0, self.shape[2])

    def scatter(self, field: torch.Tensor) -> torch.Tensor:
        """This rank's z-slab of a whole field (a copy)."""
        z0, z1 = self.z_range()
        return field[z0:z1].contiguous()


def dist_exchange(dist, group=None) -> Exchange:
    """The exchange over a torch.distributed process group: one
    all_to_all_single (NCCL all-to-all on GPUs)."""

    def exchange(send: torch.Tensor, send_counts: Sequence[int], recv_counts: Sequence[int]) -> torch.Tensor:
        recv = torch.empty(int(sum(recv_counts)), dtype=send.dtype, device=send.device)
        dist.all_to_all_single(recv, send, list(recv_counts), list(send_counts), group=group)
        return recv

    return exchange


class LocalExchange:
    """All ranks of a decomposition emulated in one process, one host thread
    per rank (``run_local``): exchange() deposits the rank's send buffer,
    waits until every rank has, and assembles what the others sent it.  The
    waits are on the host; no kernel waits on another.  For tests and
    single-GPU checks of the packing."""

    def __init__(self, size: int, timeout_s: float = 60.0):
        import threading

        self.size = size
        self.sent: list = [None] * size
        self.barrier = threading.Barrier(size, timeout=timeout_s)

    def for_rank(self, rank: int) -> Exchange:
        def exchange(send, send_counts, recv_counts):
            self.sent[rank] = (send, list(send_counts))
            self.barrier.wait()
            parts = []
            for src in range(self.size):
                buf, counts = self.sent[src]
                if counts[rank] != recv_counts[src]:
                    raise ValueError("send and receive counts disagree")
                off = sum(counts[:rank])
                parts.append(buf[off:off + counts[rank]])
            out = torch.cat(parts)
            self.barrier.wait()  # every rank has its parts before the next deposit
            return out

        return exchange


def run_local(size: int, fn: Callable[[int, Exchange], object]) -> list:
    """fn(rank, exchange) for every rank of an emulated group, each in its
    own host thread; returns the results in rank order (re-raises the first
    error)."""
    import threading

    ex = LocalExchange(size)
    results: list = [None] * size
    errors: list = []

    def body(r):
        try:
            results[r] = fn(r, ex.for_rank(r))
        except BaseException as e:  # noqa: BLE001 -- reported below
            errors.append(e)
            ex.barrier.abort()

    threads = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return results


def _z_to_y_send(s: Slabs, fz: torch.Tensor) -> tuple[torch.Tensor, list[int], list[int]]:
    nz, n2, n1 = s.z_shape()
    if tuple(fz.shape) != (nz, n2, n1) or not fz.is_contiguous():
        raise ValueError(f"expected this rank's contiguous z-slab of shape {(nz, n2, n1)}")
    send = torch.empty(fz.numel(), dtype=fz.dtype, device=fz.device)
    send_counts, off = [], 0
    for r in range(s.size):  # the y chunk for rank r, packed by one copy
        y0, y1 = s.y_range(r)
        cnt = nz * (y1 - y0) * n1
        send[off:off + cnt].view(nz, y1 - y0, n1).copy_(fz[:, y0:y1, :])
        send_counts.append(cnt)
        off += cnt
    ny = s.y_shape()[1]
    recv_counts = [s.z_shape(r)[0] * ny * n1 for r in range(s.size)]
    return send, send_counts, recv_counts


def _z_to_y_finish(s: Slabs, recv: torch.Tensor) -> torch.Tensor:
    # blocks arrive in rank order = z order, each (nz_src, ny, n1): already the y-slab
    return recv.view(s.y_shape())


def _y_to_z_send(s: Slabs, fy: torch.Tensor) -> tuple[torch.Tensor, list[int], list[int]]:
    n3, ny, n1 = s.y_shape()
    if tuple(fy.shape) != (n3, ny, n1) or not fy.is_contiguous():
        raise ValueError(f"expected this rank's contiguous y-slab of shape {(n3, ny, n1)}")
    send_counts = [(s.z_range(r)[1] - s.z_range(r)[0]) * ny * n1 for r in range(s.size)]
    nz = s.z_shape()[0]
    recv_counts = [nz * (s.y_range(r)[1] - s.y_range(r)[0]) * n1 for r in range(s.size)]
    return fy.reshape(-1), send_counts, recv_counts  # z blocks are contiguous in a y-slab


def _y_to_z_finish(s: Slabs, recv: torch.Tensor, out: torch.Tensor | None) -> torch.Tensor:
    nz, n2, n1 = s.z_shape()
    out = torch.empty((nz, n2, n1), dtype=recv.dtype, device=recv.device) if out is None else out
    off = 0
    for r in range(s.size):
        y0, y1 = s.y_range(r)
        cnt = nz * (y1 - y0) * n1
        out[:, y0:y1, :].copy_(recv[off:off + cnt].view(nz, y1 - y0, n1))
        off += cnt
    return out


def transpose_z_to_y(s: Slabs, fz: torch.Tensor, exchange: Exchange) -> torch.Tensor:
    """This rank's z-slab -> its y-slab (one all-to-all; every rank calls it)."""
    send, sc, rc = _z_to_y_send(s, fz)
    return _z_to_y_finish(s, exchange(send, sc, rc))


def transpose_y_to_z(s: Slabs, fy: torch.Tensor, exchange: Exchange,
                     out: torch.Tensor | None = None) -> torch.Tensor:
    """This rank's y-slab -> its z-slab (one all-to-all; every rank calls it);
    written into `out` when given."""
    send, sc, rc = _y_to_z_send(s, fy)
    return _y_to_z_finish(s, exchange(send, sc, rc), out)


def apply(s: Slabs, op, kind: int, axis: int, fz: torch.Tensor, dfz: torch.Tensor, exchange: Exchange,
          bc1: int = 0, bcn: int = 0, alpha: float = 1.0, beta: float = 0.0) -> None:
    """dfz = alpha * (operator `kind` of `op` along `axis`) f + beta * dfz on
    this rank's z-slabs (the distributed counterpart of der%dd*/d2d*/filter*;
    every rank calls it, with the same arguments).  x and y: local, no
    communication.  z: z-slab -> y-slab, the operator, y-slab -> z-slab."""
    nz, n2, n1 = s.z_shape()
    if axis in (1, 2):
        if nz == 0:
            return
        na, nb = (n2, nz) if axis == 1 else (n1, nz)
        op.apply(kind, axis, fz, dfz, na, nb, bc1, bcn, alpha=alpha, beta=beta)
        return
    if axis != 3:
        raise ValueError("axis must be 1, 2 or 3")
    fy = transpose_z_to_y(s, fz, exchange)
    n3, ny, _ = s.y_shape()
    dy = torch.empty_like(fy)
    if ny > 0:
        op.apply(kind, 3, fy, dy, n1, ny, bc1, bcn)
    if beta == 0.0 and alpha == 1.0:
        transpose_y_to_z(s, dy, exchange, out=dfz)
        return
    back = transpose_y_to_z(s, dy, exchange)
    if beta == 0.0:
        dfz.copy_(back).mul_(alpha)
    else:
        dfz.add_(back, alpha=alpha)


def gradient(s: Slabs, der, fz: torch.Tensor, dfdx: torch.Tensor, dfdy: torch.Tensor, dfdz: torch.Tensor,
             exchange: Exchange, x_bc=(0, 0), y_bc=(0, 0), z_bc=(0, 0)) -> None:
    """The distributed gradient (operators.F90:18-53): y and x derivatives
    on the z-slab, the z derivative through one transpose each way."""
    apply(s, der.ops[1], L.D1, 2, fz, dfdy, exchange, *y_bc)
    apply(s, der.ops[0], L.D1, 1, fz, dfdx, exchange, *x_bc)
    apply(s, der.ops[2], L.D1, 3, fz, dfdz, exchange, *z_bc)


def laplacian(s: Slabs, der, fz: torch.Tensor, lapf: torch.Tensor, exchange: Exchange,
              x_bc=(0, 0), y_bc=(0, 0), z_bc=(0, 0)) -> None:
    """The distributed laplacian (cgrid.F90:480-517), d2/dy2 + d2/dx2 +
    d2/dz2 summed in that order: the first two accumulate on the z-slab, the
    z term is added after its transpose back."""
    apply(s, der.ops[1], L.D2, 2, fz, lapf, exchange, *y_bc)
    apply(s, der.ops[0], L.D2, 1, fz, lapf, exchange, *x_bc, beta=1.0)
    apply(s, der.ops[2], L.D2, 3, fz, lapf, exchange, *z_bc, beta=1.0)
