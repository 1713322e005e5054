"""x-slab decomposition, host side: the slab geometry of splitMeshVertically
(src_WENO/fluid.cpp:99-152), and the stage / exchange order of slab_step over
torch.distributed (gloo, 3 ranks) with a host stand-in for the device
context, checked against the same stand-in over the whole grid."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from zuikakucfd_b200 import slab


def test_widths_follow_the_reference_split():
    assert slab.slab_widths(100, 3) == [33, 33, 34]  # remain // (n - k)
    assert slab.slab_widths(40, 3) == [13, 13, 14]
    assert slab.slab_widths(17, 1) == [17]
    with pytest.raises(ValueError):
        slab.slab_widths(17, 3)  # a slab of 5 columns
    with pytest.raises(ValueError):
        slab.slab_widths(40, 0)


def test_columns_and_exchange_codes():
    lay = slab.slab_columns(40, 3)
    assert [(left, w) for _, left, w in lay] == [(0, 13), (3, 13), (3, 14)]
    assert lay[0][0].tolist() == list(range(0, 16))
    assert lay[1][0].tolist() == list(range(10, 29))
    assert lay[2][0].tolist() == list(range(23, 40))
    rng = np.random.default_rng(1)
    b = np.zeros((9, 40), np.int32)
    b[:, :3] = b[:, -3:] = -1
    U = rng.standard_normal((4, 2, 9, 40))
    parts = slab.split_arrays(U, b, 3)
    for (st, bb), (cols, left, w) in zip(parts, lay):
        assert np.array_equal(st, U[..., cols])
        assert (bb[:, :left] == -3).all() and (bb[:, left + w:] == -3).all()
        assert np.array_equal(bb[:, left:left + w], b[:, cols[left:left + w]])
    assert np.array_equal(slab.join_arrays([p[0] for p in parts], 40), U)
    b[4, 20] = -3
    with pytest.raises(ValueError):
        slab.split_arrays(U, b, 3)


def test_split_mesh_vertically_copies_fields_and_options():
    from zuikakucfd_b200 import Mesh, splitMeshVertically
    rng = np.random.default_rng(2)
    m = Mesh(12, 50, 0.02, 1.4, method="dg", order=1, precision="mixed")
    m.bctype = np.where(rng.uniform(size=(12, 50)) < 0.1, -1, 0).astype(np.int32)
    m.rho, m.u, m.v, m.p = (rng.uniform(0.5, 1.0, (12, 50)) for _ in range(4))
    m.state = rng.standard_normal((4, 4, 12, 50))
    subs = splitMeshVertically(m, 3)
    assert [s.nx for s in subs] == [16 + 3, 17 + 6, 17 + 3]
    for s, (cols, left, w) in zip(subs, slab.slab_columns(50, 3)):
        assert s._opts == m._opts and (s.ny, s.da, s.gamma) == (12, 0.02, 1.4)
        assert np.array_equal(s.state, m.state[..., cols])
        assert np.array_equal(s.p, m.p[:, cols]) and np.array_equal(s.rho, m.rho[:, cols])
        assert (s.bctype[:, :left] == -3).all() and (s.bctype[:, left + w:] == -3).all()
        assert s._solver is None  # nothing touched a device
    assert np.array_equal(slab.join_arrays([s.state for s in subs], 50), m.state)


def test_slab_calls_check_the_rank_before_any_device_work():
    from zuikakucfd_b200 import Mesh, exchangeConservativeColumns, updateMesh
    m = Mesh(12, 20, 0.05, 1.4)
    for rank, n in [(1, 1), (2, 2), (-1, 3)]:
        with pytest.raises(ValueError):
            updateMesh(m, 1e-3, rank, n)
        with pytest.raises(ValueError):
            exchangeConservativeColumns(m, rank, n)
    exchangeConservativeColumns(m, 0, 1)  # one rank: nothing to exchange
    assert m._solver is None


class HostSlab:
    """Stand-in for a device context on the host: a nonlinear 7-point x
    stencil updates columns [3, nx-3) in each SSP-RK3 stage, exchange and
    ring columns are read as stored, and the 'limiter' pass smooths with the
    neighbouring columns -- so a halo sent at the wrong time changes the
    result."""

    W = (0.01, -0.05, 0.3, -0.5, 0.2, 0.03, -0.02)

    def __init__(self, U, limiter="reference"):
        self.method, self.limiter = "dg", limiter
        self.bufs = [np.array(U, np.float64), np.zeros_like(U), np.zeros_like(U)]
        self.nx = U.shape[-1]

    def _L(self, x):
        nx = self.nx
        acc = np.zeros_like(x[..., 3:nx - 3])
        for d, w in zip(range(-3, 4), self.W):
            acc = acc + w * x[..., 3 + d:nx - 3 + d]
        return acc + 0.1 * x[..., 3:nx - 3] ** 2

    def stage(self, dt, k):
        cur, un = self.bufs[k - 1], self.bufs[0]
        j = slice(3, self.nx - 3)
        L = self._L(cur)
        out = cur.copy()
        if k == 1:
            out[..., j] = un[..., j] + dt * L
        elif k == 2:
            out[..., j] = 0.75 * un[..., j] + 0.25 * (cur[..., j] + dt * L)
        else:
            out[..., j] = (1.0 / 3.0) * un[..., j] + (2.0 / 3.0) * (cur[..., j] + dt * L)
        self.bufs[k % 3] = out

    def stage_limit(self, k):
        x, nx = self.bufs[k % 3], self.nx
        y = x.copy()
        y[..., 3:nx - 3] = x[..., 3:nx - 3] + 0.05 * (x[..., 2:nx - 4] - 2 * x[..., 3:nx - 3] + x[..., 4:nx - 2])
        self.bufs[k % 3] = y

    def halo_bytes(self, k):
        return self.bufs[0][..., :3].size * 8

    def halo_pack(self, k, side, buf):
        x = self.bufs[k % 3]
        cols = slice(3, 6) if side == 0 else slice(self.nx - 6, self.nx - 3)
        nb = self.halo_bytes(k)
        buf[:nb].numpy().view(np.float64)[:] = np.ascontiguousarray(x[..., cols]).ravel()

    def halo_unpack(self, k, side, buf):
        x = self.bufs[k % 3]
        cols = slice(0, 3) if side == 0 else slice(self.nx - 3, self.nx)
        nb = self.halo_bytes(k)
        x[..., cols] = buf[:nb].numpy().view(np.float64).reshape(x[..., cols].shape)

    def max_speed(self):
        return float(np.abs(self.bufs[0][..., 3:self.nx - 3]).max())


def _initial(nx=47):
    rng = np.random.default_rng(3)
    return rng.uniform(0.5, 1.5, (4, 11, nx))


def _whole(limiter, dt, nsteps):
    h = HostSlab(_initial(), limiter)
    lam = h.max_speed()
    slab.slab_step([h], lambda k: None, dt, nsteps)
    return h.bufs[0], lam


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, limiter, out):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        U = _initial()
        st, _ = slab.split_arrays(U, np.zeros(U.shape[1:], np.int32), world)[rank]
        h = HostSlab(st, limiter)
        ex = slab.DistExchange(h, rank, world, device="cpu")
        lam = ex.max_speed()
        slab.slab_step([h], ex, 0.01, 5)
        out[rank] = (h.bufs[0], lam)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("limiter", ["reference", "tvb"])
def test_gloo_ranks_match_the_whole_grid(limiter):
    world = 3
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), limiter, out), nprocs=world, join=True)
        res = [out[r] for r in range(world)]
    ref, lam = _whole(limiter, 0.01, 5)
    got = slab.join_arrays([r[0] for r in res], ref.shape[-1])
    assert np.array_equal(got, ref)
    assert all(r[1] == lam for r in res)  # max-allreduce of the wave speed
    # the exchange matters: without it the slabs drift apart from the whole grid
    parts = [HostSlab(st, limiter) for st, _ in slab.split_arrays(_initial(), np.zeros((11, 47), np.int32), world)]
    slab.slab_step(parts, lambda k: None, 0.01, 5)
    assert not np.array_equal(slab.join_arrays([p.bufs[0] for p in parts], 47), ref)
