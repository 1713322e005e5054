"""Host side of the batched runner (no GPU): the serving workload generator."""
import numpy as np


def test_batch_problem_generator_shapes_and_split():
    from zuikakucfd_b200.batch import batch_problems
    specs = list(batch_problems(16, seed=3, sides=(16, 24, 32), nsteps=7))
    assert len(specs) == 16
    assert [s["method"] for s in specs] == ["weno"] * 8 + ["dg"] * 8
    for s in specs:
        ny, nx = s["bctype"].shape
        assert ny == nx and nx in (16, 24, 32)
        assert s["nsteps"] == 7
        if s["method"] == "dg":
            assert s["state"].shape == (4, 9, ny, nx) and s["order"] == 2
            assert not s["state"][:, 1:].any()
        else:
            assert s["state"].shape == (4, ny, nx)
    again = list(batch_problems(16, seed=3, sides=(16, 24, 32), nsteps=7))
    assert all(np.array_equal(a["state"], b["state"]) for a, b in zip(specs, again))
