"""x-slab decomposition on the GPU: a grid split into slabs (one context each,
3 exchange columns per inner side), stepped stage by stage with the halo
exchange after every stage, holds in its owned cells the same bits as one
context over the whole grid -- on every method / precision / limiter path.

The slabs share one GPU here (LocalExchange: the contexts take turns on one
stream, nothing waits on another kernel).  The rank-to-rank carrier over
torch.distributed (DistExchange) runs the same packs and unpacks around
isend/irecv; its host logic is covered by the gloo test in
test_slab_host.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PATHS = [
    ("weno", "fp64", 2, {}),
    ("weno", "mixed", 2, {}),
    ("dg", "fp64", 2, {}),
    ("dg", "fp64", 1, {"limiter": "tvb"}),
    ("dg", "mixed", 2, {}),                    # Persson + Zhang-Shu in the stage kernel
    ("dg", "mixed", 3, {"limiter": "tvb"}),    # stage kernels + TVB passes
]


def _case(method, order, seed=5):
    """Four quadrants whose x interface lies on the first slab boundary
    (columns 12 | 13 of 40), every cell perturbed so that a wrong halo
    column changes the result at once."""
    from zuikakucfd_b200 import cases
    c = cases.four_quadrant(40, seed=seed, ny=36, split=13 / 40)
    U = c.conserved()
    rng = np.random.default_rng(seed)
    U = U * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, U.shape))
    lam = c.da / cases.cfl_dt(c, 1.0)
    if method == "weno":
        return c, U, 0.4 * c.da / lam
    st = np.zeros((4, (order + 1) ** 2, c.ny, c.nx))
    st[:, 0] = U
    st[:, 1:] = 1e-3 * rng.uniform(-1.0, 1.0, st[:, 1:].shape) * U[:, None]
    return c, st, 0.5 * 0.9 / (2.0 * (2 * order + 1)) * c.da / lam


def _solver(method, precision, order, opts, ny, nx, c, bctype, state):
    from zuikakucfd_b200 import Solver
    s = Solver(method=method, order=order, precision=precision, **opts)
    s.set_mesh(ny, nx, c.da, c.gamma, bctype)
    s.set_state(state)
    return s


@pytest.mark.parametrize("nslab", [1, 3])
@pytest.mark.parametrize("method,precision,order,opts", PATHS)
def test_slabs_match_whole_grid(method, precision, order, opts, nslab):
    from zuikakucfd_b200 import slab
    c, state, dt = _case(method, order)
    nsteps = 8
    whole = _solver(method, precision, order, opts, c.ny, c.nx, c, c.bctype, state)
    lam_whole = whole.max_speed()
    whole.step(dt, nsteps)
    assert whole.status_word() == 0
    ref = whole.get_state()
    whole.close()

    parts = slab.split_arrays(state, c.bctype, nslab)
    solvers = [_solver(method, precision, order, opts, c.ny, b.shape[1], c, b, st) for st, b in parts]
    try:
        ex = slab.LocalExchange(solvers)
        assert ex.max_speed() == lam_whole          # CFL: max over the slabs
        slab.slab_step(solvers, ex, dt, nsteps)
        for s in solvers:
            assert s.status_word() == 0
        got = slab.join_arrays([s.get_state() for s in solvers], c.nx)
    finally:
        for s in solvers:
            s.close()
    assert np.isfinite(got).all()
    assert np.array_equal(got, ref)


def test_halo_pack_unpack_round_trip():
    """zk_halo_pack takes columns 3..5 / nx-6..nx-4 of the state a stage
    wrote, zk_halo_unpack writes columns 0..2 / nx-3..nx-1; FP32 halos for
    the stage states of a mixed DG context."""
    import torch
    c, state, _ = _case("dg", 2)
    s = _solver("dg", "mixed", 2, {}, c.ny, c.nx, c, c.bctype, state)
    try:
        assert s.halo_bytes(0) == 4 * 9 * c.ny * 3 * 8
        assert s.halo_bytes(1) == s.halo_bytes(2) == 4 * 9 * c.ny * 3 * 4
        buf = torch.empty(s.halo_bytes(0), dtype=torch.uint8, device="cuda")
        s.halo_pack(0, 1, buf)
        s.synchronize()
        got = buf.cpu().numpy().view(np.float64).reshape(4 * 9, c.ny, 3)
        assert np.array_equal(got, state.reshape(4 * 9, c.ny, c.nx)[:, :, c.nx - 6:c.nx - 3])
        s.halo_unpack(0, 0, buf)
        out = s.get_state().reshape(4 * 9, c.ny, c.nx)
        assert np.array_equal(out[:, :, 0:3], got)
        assert np.array_equal(out[:, :, 3:], state.reshape(4 * 9, c.ny, c.nx)[:, :, 3:])
        with pytest.raises(ValueError):
            s.halo_pack(0, 0, torch.empty(16, dtype=torch.uint8))  # host memory is refused
    finally:
        s.close()
