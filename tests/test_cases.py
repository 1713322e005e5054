"""Seeded case generator and case I/O (CPU)."""
import numpy as np

from zuikakucfd_b200 import cases
from zuikakucfd_b200.fluid import Mesh, read_case


def test_four_quadrant_conventions():
    c = cases.four_quadrant(64, seed=4)
    assert (c.ny, c.nx) == (64, 64) and c.da == 1.0 / 64
    assert c.fluid_cells == 58 * 58
    # row 0 is the top: the NE quadrant is top-right
    rng = np.random.default_rng(4)
    ne = [rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.1, 2)]
    assert c.rho[0, -1] == ne[0] and c.u[0, -1] == ne[1] and c.p[0, -1] == ne[3]
    assert c.rho[0, -1] != c.rho[-1, -1] or c.p[0, -1] != c.p[-1, -1]
    assert (c.bctype[:3] == -1).all() and (c.bctype[3:-3, 3:-3] == 0).all()
    assert c.rho.min() >= 0.1 and c.p.max() <= 2.0


def test_same_seed_same_case():
    a, b = cases.four_quadrant(32, seed=9), cases.four_quadrant(32, seed=9)
    assert np.array_equal(a.conserved(), b.conserved())
    assert not np.array_equal(a.conserved(), cases.four_quadrant(32, seed=10).conserved())


def test_smooth_wave_periodic_ring():
    w = cases.smooth_wave(32)
    assert w.periodic and w.nx == 38 and (w.bctype[:3] == -3).all()
    # the ring holds the periodic images
    assert np.array_equal(w.rho[:3, 3:-3], w.rho[-6:-3, 3:-3])
    assert np.array_equal(w.rho[3:-3, :3], w.rho[3:-3, -6:-3])
    ex = cases.smooth_wave_exact(w, 0.0)
    np.testing.assert_allclose(ex, w.rho[3:-3, 3:-3], rtol=0, atol=1e-14)
    # exact solution is periodic in t with period 1 along (1,1) / 2 ... and
    # translation by the full period returns it
    np.testing.assert_allclose(cases.smooth_wave_exact(w, 2.0), ex, atol=1e-12)


def test_jet_inflow_mechanism():
    j = cases.high_mach_jet(64, 32)
    assert (j.bctype[3:-3, :3] == 0).all() and (j.bctype[:3] == -1).all() and (j.bctype[:, -3:] == -1).all()
    band = j.rho[:, 0] == 5.0
    assert band.any() and np.all(j.u[band, :3] == 30.0) and np.all(j.u[:, 3:] == 0.0)
    assert j.gamma == 5.0 / 3.0


def test_write_then_read_case(tmp_path):
    c = cases.four_quadrant(16, seed=1, ny=12)
    cases.write_case(c, tmp_path)
    r = read_case(tmp_path)
    assert (r["nx"], r["ny"]) == (16, 12) and r["da"] == c.da and r["gamma"] == c.gamma
    for k in ("rho", "u", "v", "p", "bctype"):
        assert np.array_equal(r[k], getattr(c, k))
    m = Mesh(tmp_path)  # host side only: no device is touched until a compute call
    assert np.array_equal(m.U3, c.conserved()[3])
    md = Mesh(tmp_path, method="dg", order=2)
    assert md.dof.shape == (4, 9, 12, 16) and np.array_equal(md.dof[:, 0], c.conserved())
    assert not md.dof[:, 1:].any()
