"""zk_step runs blocks of steps as a captured CUDA graph (one eager step,
whole blocks of 16 replayed, the rest eager).  A call of many steps must give
the same bits as the same steps taken one call at a time -- for every
method / precision path -- and a changed dt is captured again."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PATHS = [
    ("weno", "fp64", 2, {}),
    ("weno", "mixed", 2, {}),
    ("dg", "fp64", 2, {}),
    ("dg", "mixed", 2, {}),                    # Persson + Zhang-Shu in the stage kernel
    ("dg", "mixed", 3, {"limiter": "tvb"}),    # stage kernels + TVB passes
]


def _case(method, order):
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(40, seed=5, ny=36)
    lam = c.da / cases.cfl_dt(c, 1.0)
    if method == "weno":
        return c, c.conserved(), 0.4 * c.da / lam
    return c, c.dg_state(order), 0.5 * 0.9 / (2.0 * (2 * order + 1)) * c.da / lam


def _run(method, precision, order, opts, calls):
    from zuikakucfd_b200 import Solver
    c, state, dt = _case(method, order)
    with Solver(method=method, order=order, precision=precision, **opts) as s:
        s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
        s.set_state(state)
        for f, n in calls:
            s.step(f * dt, n)
        assert s.status_word() == 0
        return s.get_state()


@pytest.mark.parametrize("method,precision,order,opts", PATHS)
def test_graph_steps_match_single_steps(method, precision, order, opts):
    # 40 steps: 1 eager + 2 replayed blocks + 7 eager; then a new dt: 1 + 1 block + 3
    many = _run(method, precision, order, opts, [(1.0, 40), (0.9, 20)])
    single = _run(method, precision, order, opts, [(1.0, 1)] * 40 + [(0.9, 1)] * 20)
    assert np.isfinite(many).all()
    assert np.array_equal(many, single)
