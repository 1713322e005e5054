"""GPU WENO5 mixed-precision path (FP32 reconstruction/fluxes, FP64 faces at
high Mach, FP64 accumulation) against the FP64 path and against a finer
FP64 solution (the "equal L1" criterion).

Tolerances: the mixed path is not bit-compatible; its difference from the
FP64 path on the same grid is bounded relative to the L1 norm of the field,
and its L1 error against a 4x finer FP64 solution must stay within 1.1x the
FP64 path's error.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(case, dt, steps, precision, boundary="exchange"):
    from zuikakucfd_b200 import Solver
    with Solver(method="weno", precision=precision, boundary=boundary) as s:
        s.set_mesh(case.ny, case.nx, case.da, case.gamma, case.bctype)
        s.set_state(case.conserved())
        s.step(dt, steps)
        return s.get_state(), s.status_word()


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


@pytest.mark.parametrize("n,ny,seed", [(256, 256, 1), (23, 37, 11), (100, 61, 4)])
def test_mixed_tracks_fp64(n, ny, seed):
    """Shock problems, odd sizes (TMA boxes cross the grid edge): the mixed
    state stays within 1e-5 relative L1 of the FP64 state over 50 steps."""
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(n, seed=seed, ny=ny)
    dt = cases.cfl_dt(c, 0.4)
    f64, st64 = run(c, dt, 50, "fp64")
    mix, stm = run(c, dt, 50, "mixed")
    assert st64 == 0 and stm == 0
    assert np.isfinite(mix).all()
    for q in range(4):
        assert rel_l1(mix[q], f64[q]) < 1e-5, q


def test_mixed_periodic_conserves_mass():
    from zuikakucfd_b200 import cases
    w = cases.smooth_wave(250)
    dt = 0.4 * w.da / 2.5
    mix, st = run(w, dt, 20, "mixed", boundary="periodic")
    U0 = w.conserved()
    assert st == 0
    m0, m1 = U0[0, 3:-3, 3:-3].sum(), mix[0, 3:-3, 3:-3].sum()
    assert abs(m1 - m0) / m0 < 1e-12  # FP64 accumulation of telescoping FP64-stored fluxes


def _restrict(a, f):
    """Average f x f blocks of the interior of a fine grid with a 3-cell ring."""
    x = a[3:-3, 3:-3]
    n = x.shape[0] // f
    return x.reshape(n, f, n, f).mean(axis=(1, 3))


def test_equal_l1_against_finer_fp64():
    """Four-quadrant Riemann problem at 128^2 and, as the reference solution,
    at 512^2 in FP64 (same physical time): the mixed path's density L1 error
    is <= 1.1x the FP64 path's (the metric's equal-L1 condition)."""
    from zuikakucfd_b200 import cases
    f = 4
    cc = cases.four_quadrant(128, seed=2, ring_outside=True)      # 128^2 interior on [0,1]^2
    cf = cases.four_quadrant(128 * f, seed=2, ring_outside=True)  # 512^2 interior, same states
    t_end = 0.08
    lam = 1.0 / (cases.cfl_dt(cc, 1.0) / cc.da)
    steps_c = int(np.ceil(t_end * lam / (0.4 * cc.da)))
    dt_c = t_end / steps_c
    steps_f = steps_c * f
    dt_f = t_end / steps_f
    ref, st = run(cf, dt_f, steps_f, "fp64")
    assert st == 0
    rho_ref = _restrict(ref[0], f)
    f64, _ = run(cc, dt_c, steps_c, "fp64")
    mix, _ = run(cc, dt_c, steps_c, "mixed")
    e64 = np.abs(f64[0, 3:-3, 3:-3] - rho_ref).mean()
    emx = np.abs(mix[0, 3:-3, 3:-3] - rho_ref).mean()
    assert e64 > 0
    assert emx <= 1.1 * e64, (emx, e64)


def test_high_mach_jet_positivity_and_fp64_faces():
    """Mach-80 jet at the reference's stable CFL: the mixed path (FP64 faces
    in the high-Mach band) stays positive and close to the FP64 path."""
    from zuikakucfd_b200 import cases
    j = cases.high_mach_jet(512, 256)
    dt = 0.003 * j.da / (30.0 + np.sqrt(j.gamma * 0.4127 / 5.0))
    f64, s64 = run(j, dt, 40, "fp64")
    mix, smx = run(j, dt, 40, "mixed")
    assert s64 == 0 and smx == 0
    for q in range(4):
        assert rel_l1(mix[q], f64[q]) < 1e-6, q


def test_centre_detonation_large_magnitudes():
    """The generator notebook's centre detonation (p = 1e10 Pa in a 5-cell
    charge, E ~ 2.5e10): conserved values beyond the FP32 range of the WENO
    smoothness indicators make their faces FP64, so the mixed path stays
    finite and positive and close to the FP64 path through the blast."""
    from zuikakucfd_b200 import cases
    c = cases.center_detonation(128, domain=256.0)
    dt = cases.cfl_dt(c, 0.4)
    f64, s64 = run(c, dt, 30, "fp64")
    mix, smx = run(c, dt, 30, "mixed")
    assert s64 == 0 and smx == 0
    assert np.isfinite(mix).all()
    for q in range(4):
        assert rel_l1(mix[q], f64[q]) < 1e-6, q


def test_tma_wait_timeout_is_reported_and_the_context_stays_usable():
    """The mixed WENO kernel's bounded TMA wait, made to run out without any
    fault: the barrier expects 16 bytes more than the copy delivers and the
    wait gives up after one poll.  Every CTA records STATUS_TIMEOUT, settles
    the missing bytes, lets its copy land and leaves without writing; the
    state is untouched and the next steps give the bits of a fresh context."""
    import ctypes as C
    from zuikakucfd_b200 import Solver, _native as N, cases
    c = cases.four_quadrant(64, seed=3)
    U0 = c.conserved()
    dt = cases.cfl_dt(c, 0.4)
    with Solver(method="weno", precision="mixed") as s:
        s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
        s.set_state(U0)
        st = C.c_uint32(0)
        N.check(N.lib().zk_selftest_tma_timeout(s._h, 1, C.byref(st)))
        assert st.value & 8, st.value
        assert np.array_equal(s.get_state(), U0)
        s.step(dt, 5)
        out = s.get_state()
        assert s.status_word() == 0
    ref, st2 = run(c, dt, 5, "mixed")
    assert st2 == 0
    assert np.array_equal(out, ref)
