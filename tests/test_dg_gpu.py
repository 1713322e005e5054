"""GPU DG P=1..3 FP64 path against the reference (through the C ABI).

Bar: bit-exact against the strict reference build wherever only + - * / sqrt
are involved (RHS, fluxes, CFL); the Persson filter uses log10 and sin, whose
CUDA and glibc results may differ in the last bit, so steps and the limiter are
held to 1e-12 relative L-inf against the strict build and 1e-10 against the
Makefile-faithful build.
"""
import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

CASES = [f"dg{P}_{c}" for P in (1, 2, 3) for c in ("fq20", "fq17x23", "slip22", "vacuum18")]


def solver(P, b, da, gamma, **kw):
    from zuikakucfd_b200 import Solver
    s = Solver(method="dg", order=P, **kw)
    s.set_mesh(b.shape[0], b.shape[1], da, gamma, b)
    return s


@pytest.mark.parametrize("name", CASES)
def test_dg_steps(golden, golden_meta, name):
    m = golden_meta[name]
    P = m["P"]
    d0, b = golden[f"{name}/dof0"], golden[f"{name}/bct"]
    with solver(P, b, m["da"], m["gamma"]) as s:
        s.set_state(d0)
        assert s.max_speed() == m["max_speed"]
        s.step(m["dt"], 3)
        out = s.get_state()
        assert rel_linf(out, golden[f"{name}/strict_3"]) <= 1e-12
        assert rel_linf(out, golden[f"{name}/faithful_3"]) < 1e-10
        ms = s.max_speed()
    assert abs(ms - m["max_speed_3"]) <= 1e-12 * m["max_speed_3"]


@pytest.mark.parametrize("name", CASES)
def test_dg_rhs_bit_exact_and_limiter(golden, golden_meta, name):
    m = golden_meta[name]
    P = m["P"]
    d0, b = golden[f"{name}/dof0"], golden[f"{name}/bct"]
    with solver(P, b, m["da"], m["gamma"]) as s:
        s.set_state(d0)
        dU = s.rhs(0.0)
        assert np.array_equal(dU, golden[f"{name}/rhs_dU"])
        assert np.array_equal(s.get_state(), golden[f"{name}/rhs_dof"])
        s.set_state(d0)
        s.limit()
        assert rel_linf(s.get_state(), golden[f"{name}/limit"]) <= 1e-12


@pytest.mark.parametrize("P", [1, 2, 3])
def test_dg_periodic_wave(golden, golden_meta, P):
    name = f"dg{P}_wave12"
    m = golden_meta[name]
    with solver(P, golden[f"{name}/bct"], m["da"], m["gamma"], boundary="periodic") as s:
        s.set_state(golden[f"{name}/dof0"])
        s.step(m["dt"], 3)
        out = s.get_state()
    assert rel_linf(out, golden[f"{name}/strict_3"]) <= 1e-12


@pytest.mark.parametrize("P", [1, 2, 3])
def test_dg_against_oracle_128(restatement, P):
    """128^2 seeded four-quadrant, 6 steps, GPU vs the CPU oracle; HLL flux too."""
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(128, seed=4)
    d0 = c.dg_state(P)
    lam = restatement.dg_max_speed(P, d0, c.bctype, c.gamma)
    dt = 0.5 * restatement.dg_safe_dt(P, lam, c.da)
    for flux in ("hllc", "hll"):
        ref = restatement.dg_step(P, d0, c.bctype, c.da, c.gamma, dt, 6, hll=(flux == "hll"))
        with solver(P, c.bctype, c.da, c.gamma, flux=flux) as s:
            s.set_state(d0)
            s.step(dt, 6)
            out = s.get_state()
        assert np.isfinite(ref).all()
        assert rel_linf(out, ref) <= 1e-12, flux


def test_dg_p3_full_size_determinism():
    """DG P=3 at the 2048^2 size of the learned-limiter config: two runs are
    bitwise equal and finite."""
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(2048, seed=5)
    d0 = c.dg_state(3)
    dt = 0.5 * 0.9 / 14.0 * c.da / 3.0
    outs = []
    for _ in range(2):
        with solver(3, c.bctype, c.da, c.gamma) as s:
            s.set_state(d0)
            s.step(dt, 2)
            outs.append(s.get_state())
            assert s.status_word() == 0
    assert np.array_equal(outs[0], outs[1])
    assert np.isfinite(outs[0]).all()


def test_dg_bad_options_fail_loudly():
    from zuikakucfd_b200 import Solver
    from zuikakucfd_b200._native import ZkError
    b = np.zeros((16, 16), np.int32)
    with Solver(method="dg", order=2, limiter="tvb", tvb_M=-1.0) as s:
        with pytest.raises(ZkError, match="ZK_ERR_ARG"):
            s.set_mesh(16, 16, 0.1, 1.4, b)
    with pytest.raises(ZkError, match="ZK_ERR_ARG"):
        Solver(method="dg", order=4)
