"""zk_weno_step_noalloc: the WENO5 FP64 step for callers that cannot allocate
GPU memory (their device memory belongs to another allocator, or their loop
must not pay cudaMalloc's implicit synchronisation).  The caller owns the
state and bctype buffers; the library's fixed scratch holds everything else.

Checked through the C ABI against the ordinary entry point (zk_step) with
the tolerance of the FP64 path, bit-exact equality, on two calls in a row
(two different grids, so the second call runs over the first call's leftover
scratch).  Kept in its own file, named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_steps(case, dt, steps):
    from zuikakucfd_b200 import Solver
    with Solver(method="weno", precision="fp64") as s:
        s.set_mesh(case.ny, case.nx, case.da, case.gamma, case.bctype)
        s.set_state(case.conserved())
        s.step(dt, steps)
        return s.get_state()


def _noalloc_steps(case, dt, steps, pitch):
    import torch
    from zuikakucfd_b200 import _native as N
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    U = np.zeros((4, case.ny, pitch))
    U[:, :, :case.nx] = case.conserved()
    state = torch.from_numpy(U).to(dev)                       # the caller's own buffers
    bct = torch.from_numpy(np.ascontiguousarray(case.bctype, dtype=np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    status = C.c_uint32(123)
    rc = N.lib().zk_weno_step_noalloc(
        C.cast(state.data_ptr(), C.POINTER(C.c_double)), case.ny, case.nx, pitch, case.da, case.gamma,
        C.cast(bct.data_ptr(), C.POINTER(C.c_int32)), dt, steps, C.c_void_p(stream.cuda_stream),
        C.byref(status))
    N.check(rc)
    torch.cuda.synchronize(dev)
    return state.cpu().numpy()[:, :, :case.nx], status.value


def test_noalloc_matches_zk_step_on_two_calls_in_a_row():
    from zuikakucfd_b200 import cases
    # call 1: 96 x 80 grid, odd pitch; call 2: a different grid over the same scratch
    for (n, ny, seed, steps, pitch) in [(80, 96, 3, 5, 85), (120, 64, 7, 8, 128)]:
        c = cases.four_quadrant(n, seed=seed, ny=ny)
        dt = cases.cfl_dt(c, 0.4)
        ref = _reference_steps(c, dt, steps)
        out, status = _noalloc_steps(c, dt, steps, pitch)
        assert status == 0
        assert np.array_equal(out, ref)


def test_noalloc_rejects_grids_beyond_its_scratch():
    from zuikakucfd_b200 import _native as N
    L = N.lib()
    dummy = C.cast(C.c_void_p(16), C.POINTER(C.c_double))   # never dereferenced: rejected first
    bct = C.cast(C.c_void_p(16), C.POINTER(C.c_int32))
    rc = L.zk_weno_step_noalloc(dummy, 1024, 1024, 1024, 1e-3, 1.4, bct, 1e-4, 1, None, None)
    assert rc == 1
    assert b"262144" in L.zk_last_error()
