"""The learned troubled-cell indicator fused into the mixed-precision DG stage
kernel (P=2, 3): features, tensor-core inference, the list of flagged cells
and the TVB pass over that list.  The reference has neither a TVB limiter nor
an indicator: the checks are against the project's CPU restatement of the
features, the FP32 forward pass of the network, and the plain-TVB and
unlimited paths of this library.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dg_solver(P, c, limiter, precision="mixed", **kw):
    from zuikakucfd_b200 import Solver
    s = Solver(method="dg", order=P, limiter=limiter, precision=precision, **kw)
    s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
    return s


def dg_dt(P, c, frac=0.5):
    from zuikakucfd_b200 import cases
    lam = c.da / cases.cfl_dt(c, 1.0)
    return frac * 0.9 / (2 * (2 * P + 1)) * c.da / lam


def constant_logit(value):
    """Network parameters whose logit is `value` for every input."""
    from zuikakucfd_b200 import indicator
    p = np.zeros(indicator.NPARAM, np.float32)
    p[-1] = value
    return p


def limited(s):
    from zuikakucfd_b200 import _native as N
    n = C.c_uint32()
    N.check(N.lib().zk_limited_cells(s._h, C.byref(n)))
    return n.value


def stage_logits(s, dt, stage):
    from zuikakucfd_b200 import _native as N
    n = s.ny * s.nx
    F = np.zeros((n, 40), np.float32)
    z = np.zeros(n, np.float32)
    listed = C.c_uint32()
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    N.check(N.lib().zk_indicator_stage_logits(s._h, dt, stage, fp(F), fp(z), C.byref(listed)))
    return F, z, listed.value


@pytest.mark.parametrize("P", [2, 3])
def test_every_cell_flagged_equals_plain_tvb(P):
    """A network whose logit is always positive lists every updated cell, so
    the list pass limits exactly what the plain TVB pass limits: same bits."""
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(70, seed=3, ny=45)  # partial tiles
    dt = dg_dt(P, c)
    out, counts = {}, {}
    for lim in ("tvb", "tvb_mlp"):
        with dg_solver(P, c, lim) as s:
            if lim == "tvb_mlp":
                s.set_indicator(constant_logit(1000.0))
            s.set_state(c.dg_state(P))
            total = 0
            for _ in range(6):
                s.step(dt, 1)
                total += limited(s)
            out[lim] = s.get_state()
            counts[lim] = total
            assert s.status_word() == 0
    assert counts["tvb"] > 0
    assert counts["tvb_mlp"] == counts["tvb"]
    assert np.array_equal(out["tvb_mlp"], out["tvb"])


@pytest.mark.parametrize("P", [2, 3])
def test_no_cell_flagged_equals_no_limiter(P):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(70, seed=3, ny=45)
    dt = dg_dt(P, c)
    out = {}
    for lim in ("none", "tvb_mlp"):
        with dg_solver(P, c, lim) as s:
            if lim == "tvb_mlp":
                s.set_indicator(constant_logit(-1000.0))
            s.set_state(c.dg_state(P))
            s.step(dt, 6)
            out[lim] = s.get_state()
            if lim == "tvb_mlp":
                assert limited(s) == 0
    assert np.array_equal(out["tvb_mlp"], out["none"])


def test_stage_features_and_labels_vs_restatement(restatement):
    """Training data of the indicator: features of a stage output (its modes)
    with the stage input's means, and the TVB label of the output, equal to
    the CPU restatement's (stage 1 of an unlimited FP64 step: U1 = U + dt dU)."""
    from oracle import mlp_oracle as M
    from zuikakucfd_b200 import cases, indicator
    P = 3
    c = cases.four_quadrant(30, seed=8)
    d = c.dg_state(P)
    rng = np.random.default_rng(11)
    d[:, 1:] = rng.normal(0, 0.05, d[:, 1:].shape) * np.abs(d[:, :1])
    dt = 1e-3 * c.da
    dfill, dU = restatement.dg_rhs(P, d, c.bctype, c.da, c.gamma)  # ghosts filled as the stage fills them
    s1 = dfill + dt * dU
    _, flags = restatement.dg_limit_tvb(P, s1, c.bctype, c.da, c.gamma, M=50.0)
    kind, src = restatement.ghost_map(c.bctype, with_slip=True)
    ref = M.features(P, s1, kind, src, means=d)
    with dg_solver(P, c, "none", precision="fp64") as s:
        s.set_state(d)
        s.stage(dt, 1)
        X, y = indicator.stage_features_and_labels(s, 1)
    assert flags.sum() > 10
    assert np.array_equal(y.reshape(c.ny, c.nx), flags)
    assert np.array_equal(X, ref)


def test_fused_inference_matches_fp32_forward():
    """The stage kernel's BF16 tensor-core inference against the FP32 forward
    pass on the features the kernel used; those features against the FP64
    path's features of the same stage; the list holds every positive cell."""
    from zuikakucfd_b200 import cases, indicator
    P = 3
    c = cases.four_quadrant(96, seed=9200)
    dt = dg_dt(P, c)
    w = indicator.load()
    with dg_solver(P, c, "tvb_mlp") as s:
        s.set_indicator(w)
        s.set_state(c.dg_state(P))
        s.step(dt, 8)
        st = s.get_state()
        F, z, listed = stage_logits(s, dt, 1)
    with dg_solver(P, c, "none", precision="fp64") as r:
        r.set_state(st)
        r.stage(dt, 1)
        X64, _ = indicator.stage_features_and_labels(r, 1)
    upd = np.zeros((c.ny, c.nx), bool)
    upd[3:-3, 3:-3] = c.bctype[3:-3, 3:-3] == 0
    upd = upd.ravel()
    assert np.abs(F[upd] - X64[upd]).max() < 1e-3
    assert not F[~upd].any() and not z[~upd].any()
    from oracle import mlp_oracle as M
    zt = z[upd]
    # against the FP32 forward pass (BF16 weights): the decisions; the kernel
    # also rounds features and activations to BF16, and the network's logit
    # moves by up to ~5000 per unit of a feature (it resolves the TVB
    # threshold M h^2), so single logits differ by more than the bulk
    zr = indicator.logits(w, F[upd], bf16=True)
    assert ((zt > 0) == (zr > 0)).mean() >= 0.995
    # against the same arithmetic restated on the CPU (BF16 features, weights
    # and activations): the logits themselves
    ze = M.forward_bf16(w, F[upd])
    d = np.abs(zt - ze)
    assert np.median(d) <= 1e-3 * max(1.0, np.abs(ze).max()), np.median(d)
    assert np.quantile(d, 0.99) <= 0.02 * max(1.0, np.abs(ze).max()), np.quantile(d, 0.99)
    assert ((zt > 0) == (ze > 0)).mean() >= 0.999
    assert listed == int((zt > 0).sum())
    assert listed > 0


def test_fused_indicator_step_is_faster_than_plain_tvb():
    """What the network gains in time on the metric's workload: at 2048^2,
    DG P=3 mixed, the step with the indicator fused into the stage kernel
    (TVB only on the listed cells) takes less device time than the step with
    the plain TVB pass after every stage (best of three 10-step runs each)."""
    from zuikakucfd_b200 import cases
    P = 3
    c = cases.four_quadrant(2048, seed=1000)
    dt = dg_dt(P, c)
    ms = {}
    for lim in ("tvb", "tvb_mlp"):
        with dg_solver(P, c, lim) as s:
            if lim == "tvb_mlp":
                s.set_indicator()
            s.set_state(c.dg_state(P))
            s.step(dt, 3)
            ms[lim] = min(s.step_timed(dt, 10) for _ in range(3)) / 10
            assert s.status_word() == 0
    assert ms["tvb_mlp"] < ms["tvb"], ms


def test_screen_skips_only_cells_near_a_constant_state():
    """The calibrated screen: a cell is evaluated unless every feature lies
    within the screen of a constant state's; evaluated cells get the same
    logit as without the screen, screened cells none, and only evaluated cells
    with a positive logit are listed."""
    from zuikakucfd_b200 import cases, indicator
    P = 3
    c = cases.four_quadrant(96, seed=9200)
    dt = dg_dt(P, c)
    w = indicator.load()
    tau = indicator.load_screen()
    assert tau > 0.0
    res = {}
    for screen in (-1.0, tau):
        with dg_solver(P, c, "tvb_mlp") as s:
            s.set_indicator(w, screen=screen)
            s.set_state(c.dg_state(P))
            s.step(dt, 8)
            res[screen] = stage_logits(s, dt, 1)
    (F0, z0, n0), (F1, z1, n1) = res[-1.0], res[tau]
    assert np.array_equal(F0, F1)
    upd = np.zeros((c.ny, c.nx), bool)
    upd[3:-3, 3:-3] = c.bctype[3:-3, 3:-3] == 0
    upd = upd.ravel()
    dev = indicator.deviation(F1[upd])
    ev = dev > tau
    assert ev.any() and (~ev).any()
    assert np.array_equal(z1[upd][ev], z0[upd][ev])
    assert np.isneginf(z1[upd][~ev]).all()
    assert n1 == int((z1[upd] > 0).sum()) <= n0
