"""Host-side case generation, checkpoints and result stitching (no GPU)."""
import numpy as np
import pytest


def test_riemann_config_is_the_reference_2d_riemann_case(golden):
    """The notebook's four-quadrant configuration at 256^2 with the shipped
    case's interface position reproduces the reference's 2D-Riemann input."""
    from zuikakucfd_b200 import cases
    c = cases.riemann_config(256, split=0.8)
    assert np.array_equal(c.conserved(), golden["riemann256/U0"])
    assert np.array_equal(c.bctype, golden["riemann256/bct"])


def test_center_detonation_layout():
    from zuikakucfd_b200 import cases
    c = cases.center_detonation(200, R0=50.0)
    assert (c.bctype[:2] == -1).all() and (c.bctype[:, -2:] == -1).all() and (c.bctype[2:-2, 2:-2] == 0).all()
    inside = c.p > 1e9
    # disc of radius 50 m on a 10 m grid: about pi * 5^2 cells, centred
    assert 70 <= inside.sum() <= 90
    ii, jj = np.nonzero(inside)
    assert abs(ii.mean() - 99.5) < 0.6 and abs(jj.mean() - 99.5) < 0.6
    assert np.all(c.rho[inside] == 0.1) and np.all(c.rho[~inside] == 1.225) and np.all(c.u == 0)


def test_case_cli_writes_reference_format(tmp_path):
    from zuikakucfd_b200 import cases
    from zuikakucfd_b200.fluid import read_case
    for gen in ("riemann_config", "four_quadrant", "center_detonation"):
        d = tmp_path / gen
        assert cases.main([gen, "--n", "24", "--seed", "3", "--out", str(d)]) == 0
        r = read_case(d)
        assert r["ny"] == r["nx"] == 24 and r["bctype"].dtype == np.int32
        assert np.isfinite(r["rho"]).all() and (r["rho"] > 0).all()


def test_checkpoint_round_trip(tmp_path):
    from zuikakucfd_b200 import Mesh, loadCheckpoint, saveCheckpoint
    rng = np.random.default_rng(0)
    m = Mesh(20, 30, 0.01, 1.4, method="dg", order=2, precision="mixed", limiter="tvb")
    m.bctype = rng.integers(-1, 1, (20, 30)).astype(np.int32)
    m.state = rng.standard_normal((4, 9, 20, 30))
    p = saveCheckpoint(m, tmp_path / "ck", t=0.125, step=40)
    m2, t, step = loadCheckpoint(p)
    assert (t, step) == (0.125, 40)
    assert np.array_equal(m2.state, m.state) and np.array_equal(m2.bctype, m.bctype)
    assert m2._opts == m._opts and (m2.ny, m2.nx, m2.da, m2.gamma) == (20, 30, 0.01, 1.4)
    m3, _, _ = loadCheckpoint(p, precision="fp64")
    assert m3._opts["precision"] == "fp64"


def test_combine_rank_snapshots(tmp_path):
    """Three x-slabs with 3 exchange columns each side stitch back into the
    full field (the plot notebook's rule)."""
    from zuikakucfd_b200 import combineRankSnapshots
    full = np.arange(4 * 6 * 24, dtype=float).reshape(4, 6, 24)
    cuts = [(0, 11), (5, 19), (13, 24)]  # slabs with 3-column overlaps into their neighbours
    for r, (a, b) in enumerate(cuts):
        for c in range(4):
            np.savetxt(tmp_path / f"U{c}_{r}.dat", full[c][:, a:b])
    out = combineRankSnapshots(tmp_path, 3, ghost=3)
    assert np.array_equal(out, full)
