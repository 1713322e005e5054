"""The slab schedule on the reference's own algorithm (the C restatement in
oracle/): slabs from splitMeshVertically's split, stepped stage by stage with
the 3-column exchange after every stage and limiter pass as the reference's
MPI updateMesh does (src_WENO/fluid.cpp:468-493, src_DG/fluid.cpp:1005-1054),
hold the whole-grid step's bits in their owned cells.  The schedule is run
once over the whole grid too and must give ow_step / od_step_lim's bits,
which checks the stage arithmetic restated here.

This pins the decomposition that the GPU slab path implements;
tests/test_slab_gpu.py compares that path with the GPU's whole-grid step,
which the other GPU tests compare with this restatement."""
import numpy as np
import pytest

from zuikakucfd_b200 import cases, slab


def _case(order=0, seed=7):
    c = cases.four_quadrant(40, seed=seed, ny=20, split=13 / 40)
    rng = np.random.default_rng(seed)
    U = c.conserved() * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, (4, c.ny, c.nx)))
    lam = c.da / cases.cfl_dt(c, 1.0)
    if not order:
        return c, U, 0.4 * c.da / lam
    d = np.zeros((4, (order + 1) ** 2, c.ny, c.nx))
    d[:, 0] = U
    d[:, 1:] = 1e-3 * rng.uniform(-1.0, 1.0, d[:, 1:].shape) * U[:, None]
    return c, d, 0.5 * 0.9 / (2.0 * (2 * order + 1)) * c.da / lam


def _exchange(parts, width=3):
    """exchangeColumns between neighbouring slabs, in place: the `width`
    exchange columns nearest the owned cells (3 in the reference)."""
    for a, b in zip(parts, parts[1:]):
        b[..., 3 - width:3] = a[..., -3 - width:-3]
        a[..., -3:-3 + width if width < 3 else None] = b[..., 3:3 + width]


def _combine(k, un, cur, inc):
    if k == 1:
        return un + inc
    if k == 2:
        return 0.75 * un + 0.25 * (cur + inc)
    return (1.0 / 3.0) * un + (2.0 / 3.0) * (cur + inc)


def _weno_steps(rs, parts, bcts, c, dt, nsteps, exchange=True):
    for _ in range(nsteps):
        un = [u.copy() for u in parts]
        for k in (1, 2, 3):
            nxt = []
            for u, n0, b in zip(parts, un, bcts):
                filled, dU = rs.weno_rhs(u, b, c.da, c.gamma, dt)  # dU includes dt
                nxt.append(_combine(k, n0, filled, dU))
            parts = nxt
            if exchange:
                _exchange(parts)
    return parts


def _dg_steps(rs, P, parts, bcts, c, dt, nsteps, limiter, width=3):
    for _ in range(nsteps):
        dn = [d.copy() for d in parts]
        for k in (1, 2, 3):
            nxt = []
            for d, n0, b in zip(parts, dn, bcts):
                filled, dU = rs.dg_rhs(P, d, b, c.da, c.gamma)  # d(dof)/dt
                nxt.append(_combine(k, n0, filled, dt * dU))
            parts = nxt
            if limiter == "reference":
                parts = [rs.dg_limit(P, d, b, c.gamma) for d, b in zip(parts, bcts)]
            else:  # TVB reads the neighbours' means: exchange, limit, exchange
                _exchange(parts, width)
                parts = [rs.dg_limit_tvb(P, d, b, c.da, c.gamma)[0] for d, b in zip(parts, bcts)]
            _exchange(parts, width)
    return parts


def test_weno_slabs_match_the_whole_grid_step(restatement):
    c, U, dt = _case()
    whole = restatement.weno_step(U, c.bctype, c.da, c.gamma, dt, nsteps=4)
    assert np.array_equal(_weno_steps(restatement, [U], [c.bctype], c, dt, 4)[0], whole)
    split = slab.split_arrays(U, c.bctype, 3)
    got = _weno_steps(restatement, [s for s, _ in split], [b for _, b in split], c, dt, 4)
    assert np.array_equal(slab.join_arrays(got, c.nx), whole)
    # without the exchange the slab sides drift from the whole grid
    stale = _weno_steps(restatement, [s for s, _ in split], [b for _, b in split], c, dt, 4, exchange=False)
    assert not np.array_equal(slab.join_arrays(stale, c.nx), whole)


@pytest.mark.parametrize("P,limiter", [(1, "reference"), (2, "reference"), (2, "tvb"), (3, "reference"),
                                       (3, "tvb")])
def test_dg_slabs_match_the_whole_grid_step(restatement, P, limiter):
    c, d, dt = _case(P)
    whole = restatement.dg_step_lim(P, d, c.bctype, c.da, c.gamma, dt, nsteps=2, limiter=limiter)
    assert np.array_equal(_dg_steps(restatement, P, [d], [c.bctype], c, dt, 2, limiter)[0], whole)
    split = slab.split_arrays(d, c.bctype, 3)
    got = _dg_steps(restatement, P, [s for s, _ in split], [b for _, b in split], c, dt, 2, limiter)
    assert np.array_equal(slab.join_arrays(got, c.nx), whole)


@pytest.mark.parametrize("limiter", ["reference", "tvb"])
def test_dg_needs_one_exchange_column(restatement, limiter):
    """DG reads only the face neighbour across a slab side (face fluxes and
    the TVB neighbour means), so exchanging the innermost column alone gives
    the same bits -- a third of the reference's halo bytes.  WENO's 6-point
    stencils need all three."""
    c, d, dt = _case(2)
    whole = restatement.dg_step_lim(2, d, c.bctype, c.da, c.gamma, dt, nsteps=2, limiter=limiter)
    split = slab.split_arrays(d, c.bctype, 3)
    got = _dg_steps(restatement, 2, [s for s, _ in split], [b for _, b in split], c, dt, 2, limiter, width=1)
    assert np.array_equal(slab.join_arrays(got, c.nx), whole)
    c, U, dt = _case()
    whole = restatement.weno_step(U, c.bctype, c.da, c.gamma, dt, nsteps=2)
    split = slab.split_arrays(U, c.bctype, 3)
    parts = [s_.copy() for s_, _ in split]
    for _ in range(2):
        un = [u.copy() for u in parts]
        for k in (1, 2, 3):
            parts = [_combine(k, n0, *rs_out) for n0, rs_out in
                     zip(un, (restatement.weno_rhs(u, b, c.da, c.gamma, dt) for u, (_, b) in zip(parts, split)))]
            _exchange(parts, 2)
    assert not np.array_equal(slab.join_arrays(parts, c.nx), whole)

