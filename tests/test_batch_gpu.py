"""GPU batched runner (zk_batch_*): every problem of a batch -- WENO and DG,
FP64 and mixed, of different sizes, step counts and CFL numbers, admitted by
the scheduler at different times -- ends bitwise equal to the same problem run
alone through zk_step with the time steps the batch chose; every time step
follows the reference's CFL rule applied to the max wave speed of the state
it advances; a failing problem fails alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _specs():
    from zuikakucfd_b200 import cases
    out = []
    c = cases.four_quadrant(40, seed=11, ny=56)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.conserved(), nsteps=9, cfl=0.4,
                    method="weno", precision="fp64"))
    c = cases.four_quadrant(72, seed=12, ny=61)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.conserved(), nsteps=13, cfl=0.35,
                    method="weno", precision="mixed"))
    c = cases.four_quadrant(33, seed=13)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.conserved(), nsteps=5, cfl=0.4,
                    method="weno", precision="mixed"))
    c = cases.four_quadrant(40, seed=14)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.dg_state(1), nsteps=7, cfl=0.5,
                    method="dg", order=1, precision="fp64"))
    c = cases.four_quadrant(48, seed=15, ny=37)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.dg_state(2), nsteps=11, cfl=0.5,
                    method="dg", order=2, precision="mixed"))
    c = cases.four_quadrant(36, seed=16)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.dg_state(2), nsteps=6, cfl=0.4,
                    method="dg", order=2, precision="fp64", flux="hll"))
    w = cases.smooth_wave(24)
    out.append(dict(bctype=w.bctype, da=w.da, gamma=w.gamma, state=w.dg_state(3), nsteps=8, cfl=0.5,
                    method="dg", order=3, precision="mixed", boundary="periodic"))
    c = cases.four_quadrant(30, seed=17)
    out.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.dg_state(3), nsteps=4, cfl=0.5,
                    method="dg", order=3, precision="fp64", limiter="none"))
    return out


def _single(spec, dts):
    """The same problem alone through zk_step, one step per batch dt; also
    the max wave speed (zk_max_speed) of the state before every step."""
    from zuikakucfd_b200 import Solver
    kw = {k: spec[k] for k in ("precision", "limiter", "flux", "boundary") if k in spec}
    with Solver(method=spec["method"], order=spec.get("order", 2), **kw) as s:
        b = spec["bctype"]
        s.set_mesh(b.shape[0], b.shape[1], spec["da"], spec["gamma"], b)
        s.set_state(spec["state"])
        lams = []
        for dt in dts:
            lams.append(s.max_speed())
            s.step(float(dt), 1)
        return s.get_state(), lams


def _cfl_dt(spec, lam):
    """The batch's dt rule (WENO cfl da / lambda; DG cfl * dgSafeDt)."""
    if spec["method"] == "weno":
        return spec["cfl"] * spec["da"] / lam
    P = spec["order"]
    return spec["cfl"] * (0.9 / (2.0 * (2 * P + 1)) * spec["da"] / max(lam, 1e-7))


@pytest.mark.parametrize("policy,active,gsteps", [("sjf", 3000.0, 4), ("all", 0.0, 3)])
def test_batch_matches_single_problems(policy, active, gsteps):
    from zuikakucfd_b200.batch import Batch
    specs = _specs()
    with Batch(policy=policy, active_cells=active, graph_steps=gsteps, autotune=1) as bt:
        ids = [bt.add(**s) for s in specs]
        rep = bt.run()
        assert rep["done"] == len(specs) and rep["failed"] == 0
        expect_cells = 0
        for pid, spec in zip(ids, specs):
            info = bt.info(pid)
            assert info["state"] == "done" and info["steps_done"] == spec["nsteps"], info
            assert info["status"] & 1 == 0
            dts = bt.dt_history(pid)
            assert np.all(dts > 0) and abs(info["t"] - dts.sum()) <= 1e-12 * dts.sum()
            ref, lams = _single(spec, dts)
            # every dt from the reference's max wave speed of the state it
            # advanced: the first from the reduction launch, the others from
            # the stage-3 epilogue
            assert [_cfl_dt(spec, lam) for lam in lams] == list(dts), pid
            got = bt.get_state(pid)
            assert np.array_equal(got, ref), (pid, spec["method"], spec["precision"])
            b = spec["bctype"]
            expect_cells += int((b[3:-3, 3:-3] == 0).sum()) * spec["nsteps"]
        assert rep["cell_updates"] == expect_cells
        lat = sorted(bt.info(i)["latency_ms"] for i in ids)
        assert 0 < lat[0] and rep["latency_p50_ms"] <= rep["latency_p99_ms"] <= rep["latency_max_ms"]
        assert rep["latency_max_ms"] == pytest.approx(lat[-1])
        assert rep["kernel_launches"] > 0 and rep["graph_steps"] == gsteps
        if policy == "all":
            assert rep["graph_launches"] == -(-max(s["nsteps"] for s in specs) // gsteps)
        groups = bt.groups()
        assert len(groups) == 7
        for g in groups:
            assert g["ctas_per_sm"] >= 1
            if g["method"] == "weno":
                r = g["tile_rows"]
                assert r in (4, 8) and g["tile_cols"] == 32
                assert g["threads_per_tile"] // 32 in (r // 2 + 1, r + 1, 2 * r + 2)
            elif g["precision"] == "mixed":
                assert g["tile_rows"] in (2, 4) and g["threads_per_cell"] in (1.0, 2.0)


@pytest.mark.parametrize("variant", range(6))
def test_batch_weno_tile_variants(variant):
    """Every WENO tile variant (tile height x warps per tile, pinned instead
    of tuned) gives the single-run states bit for bit."""
    from zuikakucfd_b200.batch import Batch
    specs = [s for s in _specs() if s["method"] == "weno"]
    with Batch(policy="all", graph_steps=4, autotune=1, weno_variant=variant) as bt:
        ids = [bt.add(**s) for s in specs]
        rep = bt.run()
        assert rep["done"] == len(specs)
        for pid, spec in zip(ids, specs):
            ref, _ = _single(spec, bt.dt_history(pid))
            assert np.array_equal(bt.get_state(pid), ref), (variant, spec["precision"])
        rows = (4, 8)[variant // 3]
        for g in bt.groups():
            assert g["variant"] == variant and g["tile_rows"] == rows
            assert g["threads_per_tile"] == 32 * (rows // 2 + 1, rows + 1, 2 * rows + 2)[variant % 3]


@pytest.mark.parametrize("variant", range(4))
def test_batch_dg_tile_variants(variant):
    """Every mixed DG tile variant (tile height x one or two threads per
    cell, pinned instead of tuned) gives the single-run states bit for bit,
    with the reference limiter, HLLC and periodic boundaries."""
    from zuikakucfd_b200.batch import Batch
    from zuikakucfd_b200 import cases
    specs = [s for s in _specs() if s["method"] == "dg" and s["precision"] == "mixed"]
    c = cases.four_quadrant(45, seed=18, ny=34)
    specs.append(dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.dg_state(1), nsteps=6, cfl=0.5,
                      method="dg", order=1, precision="mixed"))
    with Batch(policy="all", graph_steps=4, autotune=1, dg_variant=variant) as bt:
        ids = [bt.add(**s) for s in specs]
        rep = bt.run()
        assert rep["done"] == len(specs)
        for pid, spec in zip(ids, specs):
            ref, lams = _single(spec, bt.dt_history(pid))
            assert [_cfl_dt(spec, lam) for lam in lams] == list(bt.dt_history(pid))
            assert np.array_equal(bt.get_state(pid), ref), (variant, spec["order"])
        for g in bt.groups():
            assert g["variant"] == variant and g["tile_rows"] == (2, 4)[variant & 1]
            assert g["threads_per_cell"] == 1.0 + (variant >> 1)


def test_batch_failure_stays_local():
    """A problem driven unstable (CFL 8) fails and stops; the other finishes
    and matches its single run."""
    from zuikakucfd_b200 import cases
    from zuikakucfd_b200.batch import Batch
    good = cases.four_quadrant(48, seed=21)
    bad = cases.four_quadrant(40, seed=22)
    with Batch(policy="all", graph_steps=5, autotune=0) as bt:
        g = bt.add(good.bctype, good.da, good.gamma, good.conserved(), 20, 0.4, method="weno", precision="mixed")
        x = bt.add(bad.bctype, bad.da, bad.gamma, bad.conserved(), 60, 8.0, method="weno", precision="mixed")
        rep = bt.run()
        assert bt.info(x)["state"] == "failed" and bt.info(x)["steps_done"] < 60
        assert bt.info(g)["state"] == "done"
        assert rep["failed"] == 1 and rep["done"] == 1
        spec = dict(bctype=good.bctype, da=good.da, gamma=good.gamma, state=good.conserved(), method="weno",
                    precision="mixed")
        spec["cfl"] = 0.4
        dts = bt.dt_history(g)
        ref, lams = _single(spec, dts)
        assert [_cfl_dt(spec, lam) for lam in lams] == list(dts)
        assert np.array_equal(bt.get_state(g), ref)


def test_batch_rejects_bad_input():
    from zuikakucfd_b200 import cases
    from zuikakucfd_b200._native import ZkError
    from zuikakucfd_b200.batch import Batch
    c = cases.four_quadrant(20, seed=1)
    with Batch() as bt:
        with pytest.raises(ZkError, match="ZK_ERR_UNSUPPORTED"):
            bt.add(c.bctype, c.da, c.gamma, c.dg_state(2), 5, 0.5, method="dg", order=2, limiter="tvb")
        with pytest.raises(ZkError, match="ZK_ERR_ARG"):
            bt.add(c.bctype, c.da, c.gamma, c.conserved(), 0, 0.5)
        with pytest.raises(ZkError, match="ZK_ERR_ARG"):
            bt.add(c.bctype, c.da, c.gamma, c.conserved(), 5, -1.0)
        with pytest.raises(ZkError, match="ZK_ERR_STATE"):
            bt.run()  # empty batch
    with pytest.raises(ZkError, match="ZK_ERR_ARG"):
        Batch(weno_variant=6)
