"""GPU FP64 path with fused multiply-adds (precision "fp64_fma") against the
reference's Makefile-faithful build, which contracts a*b+c into FMAs as well.

This is the fastest plain-FP64 variant of the per-step compute (the
reference-arithmetic path is compiled with --fmad=false for bit-exactness),
so it is the denominator the mixed path's speed-up is also quoted against.
Bar: 1e-10 relative L-inf per conserved field against the faithful build
(NaN where the reference has NaN), the FP64 path's tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WENO = ["weno_fq_24x24_s3", "weno_fq_23x37_s11", "weno_fq_7x7_s5", "weno_obstacle_26",
        "weno_jet_40x20", "weno_allghost_12"]
DG = [f"dg{P}_{c}" for P in (1, 2, 3) for c in ("fq20", "fq17x23", "slip22", "vacuum18")]


def rel_linf_nan(a, b):
    """rel_linf over the finite entries; NaN / inf positions must agree."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    assert np.array_equal(fa, fb), "non-finite entries differ"
    axes = tuple(range(1, a.ndim))
    d = np.where(fb, np.abs(a - b), 0.0).max(axis=axes)
    den = np.maximum(np.where(fb, np.abs(b), 0.0).max(axis=axes), 1e-300)
    return float((d / den).max())


def solver(method, b, da, gamma, **kw):
    from zuikakucfd_b200 import Solver
    s = Solver(method=method, precision="fp64_fma", **kw)
    s.set_mesh(b.shape[0], b.shape[1], da, gamma, b)
    return s


@pytest.mark.parametrize("name", WENO)
def test_weno_fma_steps_against_faithful(golden, golden_meta, name):
    m = golden_meta[name]
    with solver("weno", golden[f"{name}/bct"], m["da"], m["gamma"]) as s:
        s.set_state(golden[f"{name}/U0"])
        s.step(m["dt"], 10)
        out = s.get_state()
    assert rel_linf_nan(out, golden[f"{name}/faithful_10"]) < 1e-10


def test_weno_fma_reference_riemann_case(golden, golden_meta):
    m = golden_meta["riemann256"]
    with solver("weno", golden["riemann256/bct"], m["da"], m["gamma"]) as s:
        s.set_state(golden["riemann256/U0"])
        s.step(m["dt"], m["steps"])
        out = s.get_state()
    assert rel_linf_nan(out[:, ::17], golden["riemann256/faithful_20_rows"]) < 1e-10


@pytest.mark.parametrize("name", DG)
def test_dg_fma_steps_against_faithful(golden, golden_meta, name):
    m = golden_meta[name]
    with solver("dg", golden[f"{name}/bct"], m["da"], m["gamma"], order=m["P"]) as s:
        s.set_state(golden[f"{name}/dof0"])
        s.step(m["dt"], 3)
        out = s.get_state()
    assert rel_linf_nan(out, golden[f"{name}/faithful_3"]) < 1e-10


@pytest.mark.parametrize("P", [2, 3])
def test_dg_fma_tvb_tracks_reference_arithmetic(P):
    """With the TVB limiter (no reference implementation to pin it), the FMA
    path stays within 1e-10 of the reference-arithmetic FP64 path over 10
    steps of a four-quadrant problem."""
    from zuikakucfd_b200 import Solver, cases
    c = cases.four_quadrant(48, seed=4)
    lam = c.da / cases.cfl_dt(c, 1.0)
    dt = 0.5 * 0.9 / (2 * (2 * P + 1)) * c.da / lam
    out = {}
    for prec in ("fp64", "fp64_fma"):
        with Solver(method="dg", order=P, precision=prec, limiter="tvb") as s:
            s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
            s.set_state(c.dg_state(P))
            s.step(dt, 10)
            out[prec] = s.get_state()
            assert s.status_word() == 0
    assert rel_linf_nan(out["fp64_fma"], out["fp64"]) < 1e-10


def test_batch_rejects_fma_precision():
    from zuikakucfd_b200 import _native as N
    from zuikakucfd_b200.batch import Batch
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(32, seed=1)
    with Batch(policy="all", graph_steps=2, autotune=0) as b:
        with pytest.raises(N.ZkError, match="precision"):
            b.add(c.bctype, c.da, c.gamma, c.conserved(), 2, 0.4, method="weno", precision="fp64_fma")
