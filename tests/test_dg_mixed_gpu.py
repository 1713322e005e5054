"""GPU DG mixed-precision path (fused FP32 stage kernel, FP64 U^n
accumulation, FP32 stage states) against the FP64 path, a finer FP64 solution
(equal L1) and the exact translated wave."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(P, case, dt, steps, precision, boundary="exchange", flux="hllc", limiter="reference", state=None):
    from zuikakucfd_b200 import Solver
    with Solver(method="dg", order=P, precision=precision, boundary=boundary, flux=flux, limiter=limiter) as s:
        s.set_mesh(case.ny, case.nx, case.da, case.gamma, case.bctype)
        s.set_state(case.dg_state(P) if state is None else state)
        s.step(dt, steps)
        return s.get_state(), s.status_word()


def dg_dt(P, case, cfl_frac=0.5):
    lam = case.da / __import__("zuikakucfd_b200").cases.cfl_dt(case, 1.0)
    return cfl_frac * 0.9 / (2.0 * (2 * P + 1)) * case.da / lam


@pytest.mark.parametrize("P", [1, 2, 3])
def test_mixed_tracks_fp64(P):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(70, seed=3, ny=45)    # odd sizes: partial tiles
    dt = dg_dt(P, c)
    f64, s1 = run(P, c, dt, 20, "fp64")
    mix, s2 = run(P, c, dt, 20, "mixed")
    assert s1 == 0 and s2 == 0
    assert np.isfinite(mix).all()
    for q in range(4):
        d = np.abs(mix[q, 0] - f64[q, 0]).sum() / np.abs(f64[q, 0]).sum()
        assert d < 2e-5, (q, d)


@pytest.mark.parametrize("P", [1, 2, 3])
def test_mixed_hll_and_no_limiter(P):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(40, seed=6)
    dt = dg_dt(P, c, 0.3)
    for flux, lim in (("hll", "reference"), ("hllc", "none")):
        f64, _ = run(P, c, dt, 10, "fp64", flux=flux, limiter=lim)
        mix, st = run(P, c, dt, 10, "mixed", flux=flux, limiter=lim)
        d = np.abs(mix[0, 0] - f64[0, 0]).sum() / np.abs(f64[0, 0]).sum()
        assert d < 2e-5, (flux, lim, d)


def _restrict(a, f):
    x = a[3:-3, 3:-3]
    n0, n1 = x.shape[0] // f, x.shape[1] // f
    return x.reshape(n0, f, n1, f).mean(axis=(1, 3))


@pytest.mark.parametrize("P", [2, 3])
def test_mixed_equal_l1_against_finer_fp64(P):
    """Four-quadrant Riemann problem: 64^2 coarse vs 256^2 FP64 reference (cell
    averages restricted), same physical time.  Mixed L1 <= 1.1 x FP64 L1."""
    from zuikakucfd_b200 import cases
    f = 4
    t_end = 0.05
    # the reference scheme (Zhang-Shu at 4x4 points with the cubic factors
    # dropped) is not positivity-preserving at P=3; use the first seed whose
    # fine FP64 reference run stays clean
    for seed in (2, 3, 5, 7, 8, 9, 10):
        cc = cases.four_quadrant(64, seed=seed, ring_outside=True)
        cf = cases.four_quadrant(64 * f, seed=seed, ring_outside=True)
        dtc = dg_dt(P, cc, 0.4)
        n = int(np.ceil(t_end / dtc))
        dtc = t_end / n
        ref, st = run(P, cf, dtc / f, n * f, "fp64")
        if st == 0:
            break
    assert st == 0
    rho_ref = _restrict(ref[0, 0], f)
    a64, _ = run(P, cc, dtc, n, "fp64")
    amx, _ = run(P, cc, dtc, n, "mixed")
    e64 = np.abs(a64[0, 0, 3:-3, 3:-3] - rho_ref).mean()
    emx = np.abs(amx[0, 0, 3:-3, 3:-3] - rho_ref).mean()
    assert emx <= 1.1 * e64, (emx, e64)


@pytest.mark.parametrize("P,limiters", [(3, ("tvb", "tvb_mlp")), (2, ("tvb",))])
def test_tvb_paths_equal_l1_against_finer_fp64(P, limiters):
    """The metric's path: DG P=3 four-quadrant Riemann problem with TVB
    limiting (M=50), mixed precision with plain TVB and with the learned
    indicator gating it, against a 4x finer FP64 + TVB solution (cell averages
    restricted, same physical time).  Each mixed path's density L1 error is at
    most 1.1 x the coarse FP64 + TVB path's."""
    from zuikakucfd_b200 import accuracy
    paths = (("fp64", "tvb"),) + tuple(("mixed", lim) for lim in limiters)
    r = accuracy.shock_refined_l1(order=P, n=64, refine=4, t_end=0.05, paths=paths)
    for key, rec in r["paths"].items():
        assert rec["status_word"] == 0, (key, rec)
    e64 = r["paths"]["fp64+tvb"]["rho_l1_err"]
    for lim in limiters:
        emx = r["paths"][f"mixed+{lim}"]["rho_l1_err"]
        assert emx <= 1.1 * e64, (lim, emx, e64, r)


def test_mixed_smooth_wave_against_exact():
    """DG P=2 periodic smooth wave at 64^2 to t=0.2: the mixed path's L1 error
    against the exact translated density is within 1.1x the FP64 path's."""
    from zuikakucfd_b200 import cases
    w = cases.smooth_wave(64)
    P = 2
    dt0 = 0.09 * w.da / 2.74
    t_end = 0.2
    n = int(np.ceil(t_end / dt0))
    dt = t_end / n
    # exact cell average of the translated wave (sin averages over a square by sinc^2)
    kh = np.pi * w.da / 2.0
    ex = 1.0 + (cases.smooth_wave_exact(w, t_end) - 1.0) * (np.sin(kh) / kh) ** 2
    errs = {}
    for prec in ("fp64", "mixed"):
        out, st = run(P, w, dt, n, prec, boundary="periodic", limiter="none")
        assert st == 0
        errs[prec] = np.abs(out[0, 0, 3:-3, 3:-3] - ex).mean()
    assert errs["mixed"] <= 1.1 * errs["fp64"], errs


def test_l2_projected_wave_convergence_and_mixed_error():
    """Smooth wave from the L2-projected start (cases.smooth_wave_modes), DG
    P=2 without limiter to t=0.1 at 32^2 and 64^2: the FP64 density error
    against the exact cell averages falls at third order.  The mixed path's
    RHS carries FP32 rounding (about 6e-8 of the flux per evaluation), so its
    error is bounded by max(1.1 x the FP64 error, 2e-7): here, far below the
    FP32 floor, the floor is what it shows."""
    from zuikakucfd_b200 import accuracy
    errs = {}
    for n in (32, 64):
        r = accuracy.run(n=n, order=2, t_end=0.1, limiter="none")
        for prec in ("fp64", "mixed"):
            assert r["paths"][prec]["status_word"] == 0
        errs[n] = (r["paths"]["fp64"]["rho_l1"], r["paths"]["mixed"]["rho_l1"])
        assert errs[n][1] <= max(1.1 * errs[n][0], 2e-7), (n, errs[n])
    order = np.log2(errs[32][0] / errs[64][0])
    assert order > 2.5, (order, errs)


@pytest.mark.parametrize("P,limiter", [(1, "reference"), (2, "tvb"), (3, "reference"), (3, "tvb")])
def test_single_path_threads_per_cell_choices_give_identical_bits(P, limiter):
    """The single-problem mixed stage with one and with two threads per cell
    (pinned through tile_tpc) and with the choice left to the autotuner gives
    the same bits; the tuner reports what it chose."""
    from zuikakucfd_b200 import Solver, cases
    c = cases.four_quadrant(70, seed=3, ny=45)
    dt = dg_dt(P, c)
    outs = {}
    for tpc in (1, 2, 0):
        with Solver(method="dg", order=P, precision="mixed", limiter=limiter, tile_tpc=tpc) as s:
            s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
            s.set_state(c.dg_state(P))
            assert s.tile_tpc() == 0
            s.step(dt, 8)
            outs[tpc] = s.get_state()
            chosen = s.tile_tpc()
            assert chosen == tpc if tpc else chosen in (1, 2)
            assert s.status_word() == 0
    assert np.array_equal(outs[1], outs[2])
    assert np.array_equal(outs[0], outs[1])


def test_fused_indicator_needs_two_threads_per_cell():
    from zuikakucfd_b200 import Solver
    from zuikakucfd_b200._native import ZkError
    with pytest.raises(ZkError, match="two threads per cell"):
        Solver(method="dg", order=3, precision="mixed", limiter="tvb_mlp", tile_tpc=1)
