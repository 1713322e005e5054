"""The headline paths at the full 2048^2 size of the metric's configuration,
through properties that hold at any size.

* Conservation.  On a periodic grid every interface flux is computed once and
  enters the two cells beside it with opposite signs, the mode-0 volume term
  is exactly zero, and neither TVB limiting nor the learned indicator's list
  pass changes a cell mean.  So the totals of the four conserved variables
  change only by rounding, in the mixed paths too.  The initial state is the
  four-quadrant state with every cell perturbed by a seeded 1e-3 relative
  factor: on the unperturbed, piecewise-constant state the FP32 rounding of
  the stored stage states is the same for every cell of a quadrant and adds
  up coherently (about 2e-8 of the totals in 5 steps); with distinct cell
  values it averages out, and the totals must hold to 1e-9.
* Determinism.  Two runs give the same bits (the indicator's list is filled
  by atomics in any order; the list pass limits each listed cell on its own).
* Agreement with the FP64 path (FMA build) after a few steps, at the
  tolerance of the mixed precision (relative L1 of density), on the
  unperturbed state for DG (limiter decisions on a field with 1e-3 jumps
  between cells differ between the learned indicator and plain TVB).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 2048
STEPS = 5


def periodic_four_quadrant(seed):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(N, seed=seed)
    c.bctype[:3, :] = -3
    c.bctype[-3:, :] = -3
    c.bctype[:, :3] = -3
    c.bctype[:, -3:] = -3
    return c


def perturbed(U, seed=11):
    """U with the cell means (mode 0) scaled by 1 + 1e-3 u, u ~ U[-1, 1] per
    cell and variable."""
    rng = np.random.default_rng(seed)
    V = U.copy()
    mean = V[:, 0] if V.ndim == 4 else V
    mean *= 1.0 + 1e-3 * rng.uniform(-1.0, 1.0, mean.shape)
    return V


def totals(U):
    """Interior totals of the cell means (mode 0 for DG) of the four variables."""
    mean = U[:, 0] if U.ndim == 4 else U
    return mean[:, 3:-3, 3:-3].sum(axis=(1, 2)), np.abs(mean[:, 3:-3, 3:-3]).sum(axis=(1, 2))


def run(method, precision, limiter, c, U0, dt, order=3):
    from zuikakucfd_b200 import Solver
    opts = dict(order=order, limiter=limiter) if method == "dg" else {}
    with Solver(method=method, precision=precision, boundary="periodic", **opts) as s:
        s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
        if limiter == "tvb_mlp":
            s.set_indicator()
        s.set_state(U0)
        s.step(dt, STEPS)
        out = s.get_state()
        assert s.status_word() == 0
    return out


def test_dg_p3_mixed_learned_indicator_full_size():
    from zuikakucfd_b200 import cases
    c = periodic_four_quadrant(seed=1000)
    dt = 0.5 * 0.9 / 14.0 * cases.cfl_dt(c, 1.0)
    # conservation and determinism on the perturbed state
    U0 = perturbed(c.dg_state(3))
    t0, s0 = totals(U0)
    a = run("dg", "mixed", "tvb_mlp", c, U0, dt)
    b = run("dg", "mixed", "tvb_mlp", c, U0, dt)
    assert np.array_equal(a, b), "two runs of the headline path differ"
    t1, _ = totals(a)
    assert np.all(np.abs(t1 - t0) <= 1e-9 * s0), (t1 - t0) / s0
    assert not np.array_equal(a[:, 0], U0[:, 0])
    del a, b
    f = run("dg", "fp64_fma", "tvb", c, U0, dt)
    tf, _ = totals(f)
    assert np.all(np.abs(tf - t0) <= 1e-12 * s0), (tf - t0) / s0
    del f, U0
    # agreement with the FP64 path on the four-quadrant state itself (on the
    # perturbed one, whose cells jump by 1e-3, the learned indicator and the
    # plain TVB test limit some cells differently)
    U0 = c.dg_state(3)
    m = run("dg", "mixed", "tvb_mlp", c, U0, dt)[0, 0, 3:-3, 3:-3]
    f = run("dg", "fp64_fma", "tvb", c, U0, dt)[0, 0, 3:-3, 3:-3]
    d = np.abs(m - f)
    assert d.sum() / np.abs(f).sum() < 1e-6
    assert d.max() / np.abs(f).max() < 1e-3


def test_weno_mixed_full_size():
    from zuikakucfd_b200 import cases
    c = periodic_four_quadrant(seed=1000)
    U0 = perturbed(c.conserved())
    dt = cases.cfl_dt(c, 0.4)
    a = run("weno", "mixed", None, c, U0, dt)
    b = run("weno", "mixed", None, c, U0, dt)
    assert np.array_equal(a, b)
    t0, s0 = totals(U0)
    t1, _ = totals(a)
    # interface fluxes are FP64 in shared memory, dU and the combine FP64
    assert np.all(np.abs(t1 - t0) <= 1e-12 * s0), (t1 - t0) / s0
    f = run("weno", "fp64_fma", None, c, U0, dt)
    d = np.abs(a[0, 3:-3, 3:-3] - f[0, 3:-3, 3:-3])
    assert d.sum() / np.abs(f[0, 3:-3, 3:-3]).sum() < 1e-6
