"""GPU post-processing: the Mach number field (the plot notebook's
compute_mach) against numpy on the recovered primitives, WENO and DG."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,order", [("weno", 2), ("dg", 2)])
def test_mach_number_matches_primitives(method, order):
    from zuikakucfd_b200 import Mesh, cases, computeMach, recoverPrimitives
    c = cases.four_quadrant(40, seed=2, ny=33)
    m = Mesh(c.ny, c.nx, c.da, c.gamma, method=method, order=order)
    m.bctype = c.bctype
    m.state = c.conserved() if method == "weno" else c.dg_state(order)
    mach, speed = computeMach(m)
    recoverPrimitives(m)
    vel = np.sqrt(m.u ** 2 + m.v ** 2)
    np.testing.assert_allclose(speed, vel, rtol=1e-14, atol=0)
    np.testing.assert_allclose(mach, vel / np.sqrt(c.gamma * m.p / m.rho), rtol=1e-14, atol=1e-300)
    m.close()
