"""TVB limiter (Cockburn-Shu TVB minmod, characteristic) and the learned
indicator on the GPU, against the project's CPU restatements.  The reference
has no TVB limiter and no indicator: parity is against the restatements only
(unpinned by the reference)."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu


def dg_solver(P, c, limiter, precision="fp64", **kw):
    from zuikakucfd_b200 import Solver
    s = Solver(method="dg", order=P, limiter=limiter, precision=precision, **kw)
    s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
    return s


def rough_state(P, c, seed):
    d = c.dg_state(P)
    rng = np.random.default_rng(seed)
    d[:, 1:] = rng.normal(0, 0.05, d[:, 1:].shape) * np.abs(d[:, :1])
    return d


@pytest.mark.parametrize("P", [1, 2, 3])
def test_tvb_pass_bit_exact_vs_restatement(restatement, P):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(40, seed=4, ny=33)
    d = rough_state(P, c, P)
    ref, flags = restatement.dg_limit_tvb(P, d, c.bctype, c.da, c.gamma, M=50.0)
    assert flags.sum() > 10
    with dg_solver(P, c, "tvb") as s:
        s.set_state(d)
        s.limit()
        out = s.get_state()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("P", [1, 2, 3])
def test_tvb_steps_vs_restatement(restatement, P):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(48, seed=6)
    d0 = c.dg_state(P)
    lam = restatement.dg_max_speed(P, d0, c.bctype, c.gamma)
    dt = 0.5 * restatement.dg_safe_dt(P, lam, c.da)
    ref = restatement.dg_step_lim(P, d0, c.bctype, c.da, c.gamma, dt, 4, limiter="tvb", M=50.0)
    with dg_solver(P, c, "tvb") as s:
        s.set_state(d0)
        s.step(dt, 4)
        out = s.get_state()
    assert np.isfinite(ref).all()
    assert rel_linf(out, ref) <= 1e-12
    with dg_solver(P, c, "tvb", precision="mixed") as s:
        s.set_state(d0)
        s.step(dt, 4)
        mix = s.get_state()
    assert np.abs(mix[0, 0] - ref[0, 0]).sum() / np.abs(ref[0, 0]).sum() < 1e-4


def test_features_and_labels_vs_restatement(restatement):
    from oracle import mlp_oracle as M
    from zuikakucfd_b200 import cases, indicator
    P = 3
    c = cases.four_quadrant(30, seed=8)
    d = rough_state(P, c, 11)
    _, flags = restatement.dg_limit_tvb(P, d, c.bctype, c.da, c.gamma, M=50.0)
    kind, src = restatement.ghost_map(c.bctype, with_slip=True)
    ref = M.features(P, d, kind, src)
    with dg_solver(P, c, "tvb") as s:
        s.set_state(d)
        X, y = indicator.features_and_labels(s)
        assert np.array_equal(s.get_state(), d)  # extraction does not touch the state
    assert np.array_equal(y.reshape(c.ny, c.nx), flags)
    assert np.array_equal(X, ref)


def test_mlp_gradient_and_forward_vs_oracle():
    from oracle import mlp_oracle as M
    from zuikakucfd_b200 import _native as N
    rng = np.random.default_rng(1)
    p = M.init_params(5)
    X = rng.normal(0, 1, (300, M.IN)).astype(np.float32)
    y = (rng.random(300) < 0.2).astype(np.uint8)
    g = np.zeros(M.NPARAM, np.float32)
    loss = C.c_float()
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    N.check(N.lib().zk_mlp_grad(0, fp(X), y.ctypes.data_as(C.POINTER(C.c_uint8)), len(y), fp(p), 3.0, fp(g),
                                C.byref(loss)))
    lref, gref = M.loss_and_grad(p, X, y, 3.0)
    assert abs(loss.value - lref) <= 1e-5 * abs(lref)
    assert np.abs(g - gref).max() <= 1e-4 * np.abs(gref).max()
    from zuikakucfd_b200 import indicator
    z = indicator.logits(p, X, bf16=False)
    zr, _ = M.forward(p, X)
    assert np.abs(z - zr).max() <= 1e-4 * max(1.0, np.abs(zr).max())


def test_training_learns_a_separable_rule():
    from zuikakucfd_b200 import indicator
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (40_000, 40)).astype(np.float32)
    y = ((X[:, 0] + 0.5 * X[:, 33] - X[:, 36]) > 1.2).astype(np.uint8)
    p, losses = indicator.train(X, y, epochs=8, batch=1024, lr=3e-3, seed=1)
    assert losses[-1] < 0.5 * losses[0]
    ag = indicator.agreement(p, X, y)
    assert ag["accuracy"] > 0.97 and ag["missed_rate"] < 0.1


def test_shipped_indicator_gates_tvb_limiting():
    """The trained indicator (zuikakucfd_b200/data/indicator_p3.npz) on a
    held-out seed: the gated run limits cells close to where plain TVB does,
    stays finite and positive, and its solution is close to the plain-TVB
    run; an unlimited run of the same case is the contrast."""
    from zuikakucfd_b200 import _native as N, cases, indicator
    P = 3
    c = cases.four_quadrant(256, seed=9100)
    lam = c.da / cases.cfl_dt(c, 1.0)
    dt = 0.5 * 0.9 / (2 * (2 * P + 1)) * c.da / lam
    w = indicator.load()
    runs, counts = {}, {}
    for lim in ("tvb", "tvb_mlp", "none"):
        with dg_solver(P, c, lim, precision="mixed") as s:
            if lim == "tvb_mlp":
                N.check(N.lib().zk_set_indicator(s._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))
            s.set_state(c.dg_state(P))
            total = 0
            for _ in range(10):
                s.step(dt, 6)
                n = C.c_uint32()
                N.check(N.lib().zk_limited_cells(s._h, C.byref(n)))
                total += n.value
            runs[lim] = (s.get_state(), s.status_word())
            counts[lim] = total
    tvb, st_t = runs["tvb"]
    mlp, st_m = runs["tvb_mlp"]
    assert st_t == 0 and st_m == 0
    assert np.isfinite(mlp).all() and mlp[0, 0, 3:-3, 3:-3].min() > 0
    assert counts["tvb_mlp"] > 0.5 * counts["tvb"]
    d = np.abs(mlp[0, 0] - tvb[0, 0]).sum() / np.abs(tvb[0, 0]).sum()
    assert d < 5e-3, d


def test_indicator_requires_weights():
    from zuikakucfd_b200 import cases
    from zuikakucfd_b200._native import ZkError
    c = cases.four_quadrant(32, seed=1)
    with dg_solver(3, c, "tvb_mlp") as s:
        s.set_state(c.dg_state(3))
        with pytest.raises(ZkError, match="indicator weights not set"):
            s.step(1e-4, 1)


def test_tensor_core_inference_matches_fp32_forward():
    """The limiter's BF16 mma.sync inference against the FP32 forward pass on
    the same features: logits close, decisions agree."""
    from zuikakucfd_b200 import _native as N, cases, indicator
    P = 3
    c = cases.four_quadrant(96, seed=9200)
    lam = c.da / cases.cfl_dt(c, 1.0)
    dt = 0.5 * 0.9 / (2 * (2 * P + 1)) * c.da / lam
    w = indicator.load()
    with dg_solver(P, c, "tvb_mlp") as s:
        N.check(N.lib().zk_set_indicator(s._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))
        s.set_state(c.dg_state(P))
        s.step(dt, 8)
        X, y = indicator.features_and_labels(s)
        z = np.zeros(c.ny * c.nx, np.float32)
        N.check(N.lib().zk_indicator_logits(s._h, z.ctypes.data_as(C.POINTER(C.c_float))))
    upd = np.zeros((c.ny, c.nx), bool)
    upd[3:-3, 3:-3] = True
    upd = upd.ravel()
    zr = indicator.logits(w, X[upd], bf16=True)
    zt = z[upd]
    assert np.abs(zt - zr).max() <= 0.05 * max(1.0, np.abs(zr).max())
    assert ((zt > 0) == (zr > 0)).mean() >= 0.995
