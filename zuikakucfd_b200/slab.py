"""x-slab decomposition of one grid over several device contexts.

The reference's MPI runs split the grid into vertical slabs
(splitMeshVertically, src_WENO/fluid.cpp:99-152 and src_DG/fluid.cpp:249-312),
give every inner slab side 3 exchange columns (bctype -3), swap 3 columns per
field with each neighbour after every RK stage and limiter pass
(exchangeConservativeColumns, src_WENO/fluid.cpp:160-198 and 468-493;
src_DG/fluid.cpp:342-400 and 1005-1054) and take the max of the ranks' wave
speeds for dt (MPI_Allreduce MAX, src_WENO/solver.cpp:146-170).

Here a slab is one ``Solver`` (one ``zk_ctx``); a step is the three stage
kernels of ``zk_step`` run one at a time (``zk_stage``), each followed by a
halo exchange: the native ``zk_halo_pack`` copies the 3 owned columns next to
an inner side into a contiguous device buffer, the buffer crosses to the
neighbour, and ``zk_halo_unpack`` stores it in the neighbour's exchange
columns.  Two carriers move the buffers:

* ``DistExchange``: one slab per rank of a ``torch.distributed`` group
  (NCCL between GPUs, gloo for host buffers), isend/irecv with the left and
  right ranks; the context and the NCCL calls share one stream, so the pack,
  the transfer and the unpack are ordered on the device.
* ``LocalExchange``: every slab in one process on one device, buffers handed
  from one context to the next on a single stream.

The owned cells of the slabs hold the bits that one context over the whole
grid computes (the same kernels read the same stencil values).
"""
from __future__ import annotations

import contextlib
from typing import Callable, Sequence

import numpy as np

GHOST = 3  # exchange columns per inner side (WENO5 stencil half-width)
MIN_WIDTH = 2 * GHOST  # owned columns a slab needs: sources of its ring, halos of its neighbours


def slab_widths(nx: int, n: int) -> list[int]:
    """Owned columns of each of n slabs: widths[k] = remain // (n - k), as
    splitMeshVertically (src_WENO/fluid.cpp:103-105) divides them."""
    if n < 1:
        raise ValueError("need at least one slab")
    widths, remain = [], int(nx)
    for k in range(n):
        w = remain // (n - k)
        widths.append(w)
        remain -= w
    if n > 1 and min(widths) < MIN_WIDTH:
        raise ValueError(f"{nx} columns over {n} slabs leaves a slab narrower than {MIN_WIDTH} columns")
    return widths


def slab_columns(nx: int, n: int) -> list[tuple[np.ndarray, int, int]]:
    """Per slab: (source column of every local column, first owned local
    column, owned width).  Exchange columns take the neighbour's columns,
    clamped to the grid (src_WENO/fluid.cpp:126-145)."""
    out, start = [], 0
    for k, w in enumerate(slab_widths(nx, n)):
        left = GHOST if k > 0 else 0
        right = GHOST if k < n - 1 else 0
        cols = [max(start - left + g, 0) for g in range(left)]
        cols += list(range(start, start + w))
        cols += [min(start + w + g, nx - 1) for g in range(right)]
        out.append((np.asarray(cols, np.int64), left, w))
        start += w
    return out


def split_arrays(state: np.ndarray, bctype: np.ndarray, n: int) -> list[tuple[np.ndarray, np.ndarray]]:
    """(state, bctype) of each slab; state's last axis is x.  The exchange
    columns copy the neighbour's values and get bctype -3."""
    bctype = np.asarray(bctype, np.int32)
    if np.any(bctype == -3):
        raise ValueError("the grid already has exchange (-3) cells: periodic rings are not split")
    parts = []
    for cols, left, w in slab_columns(bctype.shape[1], n):
        b = bctype[:, cols].copy()
        b[:, :left] = -3
        b[:, left + w:] = -3
        parts.append((np.ascontiguousarray(state[..., cols]), b))
    return parts


def join_arrays(parts: Sequence[np.ndarray], nx: int) -> np.ndarray:
    """The whole-grid array from the slabs' arrays (owned columns only)."""
    layout = slab_columns(nx, len(parts))
    return np.concatenate([p[..., left:left + w] for p, (_, left, w) in zip(parts, layout)], axis=-1)


def _tvb(solver) -> bool:
    return solver.method == "dg" and getattr(solver, "limiter", "reference") in ("tvb", "tvb_mlp")


class LocalExchange:
    """Halo exchange between slabs that all live in this process on one
    device.  Every context is moved onto one stream, so each pack, unpack and
    stage is ordered after the one before it."""

    def __init__(self, solvers: Sequence, stream=None):
        import torch
        devs = {s.device for s in solvers}
        if len(devs) != 1:
            raise ValueError("LocalExchange keeps every slab on one device")
        self.solvers = list(solvers)
        dev = torch.device("cuda", devs.pop())
        # a stream of its own: a null handle would send each context back to its own stream
        self.stream = stream if stream is not None else torch.cuda.Stream(dev)
        if not self.stream.cuda_stream:
            raise ValueError("LocalExchange needs a non-default stream")
        for s in self.solvers:
            s.set_stream(self.stream.cuda_stream)
        nb = max(s.halo_bytes(k) for s in self.solvers for k in range(4))
        self.buf = torch.empty(nb, dtype=torch.uint8, device=dev)

    def __call__(self, stage: int) -> None:
        b = self.buf
        for a, c in zip(self.solvers, self.solvers[1:]):
            a.halo_pack(stage, 1, b)    # a's last owned columns -> c's left exchange columns
            c.halo_unpack(stage, 0, b)
            c.halo_pack(stage, 0, b)    # c's first owned columns -> a's right exchange columns
            a.halo_unpack(stage, 1, b)

    def max_speed(self) -> float:
        return max(s.max_speed() for s in self.solvers)


class DistExchange:
    """Halo exchange of this rank's slab with ranks rank-1 and rank+1 of a
    torch.distributed group (ranks of the default group).  Device slabs use
    the group's NCCL backend on a stream the context shares; host slabs
    (buffers on the CPU) use gloo."""

    def __init__(self, solver, rank: int, nprocs: int, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.solver, self.rank, self.nprocs, self.group = solver, int(rank), int(nprocs), group
        if device is None:
            device = torch.device("cuda", solver.device)
        self.device = torch.device(device)
        self.stream = None
        if self.device.type == "cuda":
            # the context, the packs and the NCCL calls share this stream
            self.stream = torch.cuda.Stream(self.device)
            solver.set_stream(self.stream.cuda_stream)
        nb = max(solver.halo_bytes(k) for k in range(4))
        with self._on_stream():
            self.send = [torch.empty(nb, dtype=torch.uint8, device=self.device) for _ in range(2)]
            self.recv = [torch.empty(nb, dtype=torch.uint8, device=self.device) for _ in range(2)]
            # every rank joins one collective before the first point-to-point call
            flag = torch.ones(1, device=self.device)
            dist.all_reduce(flag, group=group)

    def _on_stream(self):
        import torch
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def _peer(self, side: int) -> int | None:
        p = self.rank - 1 if side == 0 else self.rank + 1
        return p if 0 <= p < self.nprocs else None

    def __call__(self, stage: int) -> None:
        import torch.distributed as dist
        s = self.solver
        nb = s.halo_bytes(stage)
        ops = []
        for side in (0, 1):
            peer = self._peer(side)
            if peer is None:
                continue
            s.halo_pack(stage, side, self.send[side])
            ops.append(dist.P2POp(dist.isend, self.send[side][:nb], peer, self.group))
            ops.append(dist.P2POp(dist.irecv, self.recv[side][:nb], peer, self.group))
        if not ops:
            return
        with self._on_stream():
            for w in dist.batch_isend_irecv(ops):
                w.wait()  # NCCL: the stream waits; gloo: the host waits
        for side in (0, 1):
            if self._peer(side) is not None:
                s.halo_unpack(stage, side, self.recv[side])

    def max_speed(self) -> float:
        import torch
        import torch.distributed as dist
        with self._on_stream():
            v = torch.tensor([self.solver.max_speed()], dtype=torch.float64, device=self.device)
            dist.all_reduce(v, op=dist.ReduceOp.MAX, group=self.group)
            return float(v.item())


def slab_step(solvers: Sequence, exchange: Callable[[int], None], dt: float, nsteps: int = 1) -> None:
    """nsteps SSP-RK3 steps of slabs: for each stage, the stage kernels of
    every local slab, then the exchange; DG TVB limiters add the limiter pass
    between two exchanges (src_DG/fluid.cpp:1020-1053: limit, then exchange)."""
    tvb = _tvb(solvers[0])
    for _ in range(int(nsteps)):
        for k in (1, 2, 3):
            for s in solvers:
                s.stage(dt, k)
            if tvb:
                exchange(k)
                for s in solvers:
                    s.stage_limit(k)
            exchange(k)
