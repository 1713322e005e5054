"""Host-side mirror of ZuikakuCFD's solver interface over the C ABI.

The reference exposes plain C++ free functions over a ``Mesh`` object
(src_WENO/fluid.h, src_DG/fluid.h).  This module keeps those names, argument
meanings and in-place semantics, with the compute on the GPU:

    mesh = Mesh("2D-Riemann")                 # Mesh(folder)
    lam  = computeMaxSpeed(mesh, mesh.gamma)  # src_WENO/fluid.cpp:539
    updateMesh(mesh, dt, 0, 1)                # src_WENO/fluid.cpp:468 (one SSP-RK3 step)
    dU   = computeRHS(mesh, dt)               # src_WENO/fluid.cpp:328 (fills ghosts in place)
    recoverPrimitives(mesh)                   # src_WENO/fluid.cpp:500

The conserved state lives on the device between calls; the host arrays
(``U0..U3``, ``dof``) are refreshed lazily when read, and host writes are
pushed before the next device call.  Array layout is row-major ``[ny, nx]``
with row 0 on top, indexed ``mesh.U0[i, j]`` like the reference's ``U0(i, j)``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import _native as N


class Solver:
    """One device context (``zk_ctx``): device-resident state and a CUDA stream."""

    def __init__(self, method: str = "weno", order: int = 2, precision: str = "fp64",
                 limiter: str = "reference", flux: str = "hllc", boundary: str = "exchange",
                 device: int = 0, tvb_M: float = 50.0, recon: str = "weno5", tile_tpc: int = 0):
        L = N.lib()
        o = N.zk_options()
        L.zk_default_options(C.byref(o))
        o.method = N.METHOD[method]
        o.order = int(order)
        o.precision = N.PRECISION[precision]
        o.limiter = N.LIMITER[limiter]
        o.flux = N.FLUX[flux]
        o.boundary = N.BOUNDARY[boundary]
        o.device = int(device)
        o.tvb_M = float(tvb_M)
        o.recon = N.RECON[recon]
        o.tile_tpc = int(tile_tpc)
        h = C.c_void_p()
        N.check(L.zk_create(C.byref(o), C.byref(h)))
        self._h = h
        self.method, self.order, self.precision = method, int(order), precision
        self.limiter, self.device = limiter, int(device)
        self.nm = (self.order + 1) ** 2 if method == "dg" else 1
        self.ny = self.nx = 0

    # -- lifetime ---------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().zk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- mesh / state --------------------------------------------------------------
    @property
    def state_shape(self) -> tuple:
        if self.method == "dg":
            return (4, self.nm, self.ny, self.nx)
        return (4, self.ny, self.nx)

    def set_mesh(self, ny: int, nx: int, da: float, gamma: float, bctype) -> None:
        b = np.ascontiguousarray(bctype, dtype=np.int32)
        if b.shape != (ny, nx):
            raise ValueError(f"bctype shape {b.shape} != ({ny}, {nx})")
        N.check(N.lib().zk_set_mesh(self._h, int(ny), int(nx), float(da), float(gamma),
                                    b.ctypes.data_as(C.POINTER(C.c_int32))))
        self.ny, self.nx = int(ny), int(nx)

    def load_case(self, folder: str | os.PathLike) -> None:
        N.check(N.lib().zk_load_case(self._h, str(folder).encode()))
        p = Path(folder, "params.txt").read_text().split()
        self.nx, self.ny = int(p[0]), int(p[1])

    def set_state(self, state) -> None:
        s = np.ascontiguousarray(state, dtype=np.float64)
        if s.shape != self.state_shape:
            raise ValueError(f"state shape {s.shape} != {self.state_shape}")
        N.check(N.lib().zk_set_state(self._h, N.dptr(s)))

    def get_state(self) -> np.ndarray:
        out = np.empty(self.state_shape, dtype=np.float64)
        N.check(N.lib().zk_get_state(self._h, N.dptr(out)))
        return out

    # -- compute -------------------------------------------------------------------
    def step(self, dt: float, nsteps: int = 1) -> None:
        N.check(N.lib().zk_step(self._h, float(dt), int(nsteps)))

    def step_timed(self, dt: float, nsteps: int) -> float:
        ms = C.c_float()
        N.check(N.lib().zk_step_timed(self._h, float(dt), int(nsteps), C.byref(ms)))
        return float(ms.value)

    def rhs(self, dt: float) -> np.ndarray:
        out = np.empty(self.state_shape, dtype=np.float64)
        N.check(N.lib().zk_rhs(self._h, float(dt), N.dptr(out)))
        return out

    def limit(self) -> None:
        N.check(N.lib().zk_limit(self._h))

    def max_speed(self) -> float:
        v = C.c_double()
        N.check(N.lib().zk_max_speed(self._h, C.byref(v)))
        return float(v.value)

    def recover_primitives(self) -> np.ndarray:
        out = np.empty((4, self.ny, self.nx), dtype=np.float64)
        N.check(N.lib().zk_recover_primitives(self._h, N.dptr(out)))
        return out

    def set_indicator(self, params=None, screen: float | None = None) -> None:
        """Weights of the learned troubled-cell indicator (limiter "tvb_mlp"):
        a flat FP32 block of MLP_NPARAM values; None loads the trained weights
        shipped with the package together with their calibrated screen
        (zk_set_indicator_screen).  `screen` overrides it (< 0: none)."""
        from . import indicator
        w = np.ascontiguousarray(indicator.load() if params is None else params, np.float32)
        N.check(N.lib().zk_set_indicator(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))
        if screen is None:
            screen = indicator.load_screen() if params is None else -1.0
        N.check(N.lib().zk_set_indicator_screen(self._h, float(screen)))

    def tile_tpc(self) -> int:
        """Threads per cell of the mixed DG stage kernel (0 before the first step)."""
        v = C.c_int()
        N.check(N.lib().zk_tile_tpc(self._h, C.byref(v)))
        return int(v.value)

    def status_word(self) -> int:
        v = C.c_uint32()
        N.check(N.lib().zk_status_word(self._h, C.byref(v)))
        return int(v.value)

    def synchronize(self) -> None:
        N.check(N.lib().zk_synchronize(self._h))

    def set_stream(self, stream_handle: int | None) -> None:
        N.check(N.lib().zk_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    # -- one stage at a time and slab halos (zuikakucfd_b200.slab) ------------------
    def stage(self, dt: float, stage: int) -> None:
        """Enqueue stage 1, 2 or 3 of one step (the kernels zk_step runs)."""
        N.check(N.lib().zk_stage(self._h, float(dt), int(stage)))

    def stage_limit(self, stage: int) -> None:
        """Enqueue the TVB pass that follows `stage` (no-op for other limiters)."""
        N.check(N.lib().zk_stage_limit(self._h, int(stage)))

    def halo_bytes(self, stage: int) -> int:
        v = C.c_size_t()
        N.check(N.lib().zk_halo_bytes(self._h, int(stage), C.byref(v)))
        return int(v.value)

    def halo_pack(self, stage: int, side: int, buf) -> None:
        """Copy the 3 owned columns next to `side` (0 left, 1 right) of the
        state `stage` wrote into `buf`, a device tensor on this context's
        device of at least halo_bytes(stage) bytes."""
        N.check(N.lib().zk_halo_pack(self._h, int(stage), int(side), C.c_void_p(_device_ptr(buf, self.device))))

    def halo_unpack(self, stage: int, side: int, buf) -> None:
        """Store `buf` (as packed by the neighbour) in the exchange columns of `side`."""
        N.check(N.lib().zk_halo_unpack(self._h, int(stage), int(side), C.c_void_p(_device_ptr(buf, self.device))))


def _device_ptr(buf, device: int) -> int:
    """Address of a CUDA tensor on `device`; anything else is refused, since
    the halo kernels dereference it on the GPU."""
    dev = getattr(buf, "device", None)
    if dev is None or dev.type != "cuda" or dev.index != device:
        raise ValueError(f"halo buffer must be a CUDA tensor on cuda:{device}")
    return int(buf.data_ptr())


# ---------------------------------------------------------------------------------
# Reference-shaped API
# ---------------------------------------------------------------------------------

def read_case(folder: str | os.PathLike) -> dict:
    """Parse params.txt ("nx ny da gamma") and the row-major rho/u/v/p/bctype
    .dat files of a case directory (src_WENO/fluid.cpp:33-94)."""
    folder = Path(folder)
    try:
        p = (folder / "params.txt").read_text().split()
    except OSError as e:
        raise RuntimeError("Cannot open params.txt") from e
    nx, ny, da, gamma = int(p[0]), int(p[1]), float(p[2]), float(p[3])
    out = {"nx": nx, "ny": ny, "da": da, "gamma": gamma}
    for name in ("rho", "u", "v", "p", "bctype"):
        f = folder / f"{name}.dat"
        if not f.exists():
            raise RuntimeError(f"Cannot open file: {f}")
        dt = np.int32 if name == "bctype" else np.float64
        a = np.loadtxt(f, dtype=dt, ndmin=2)
        if a.size != ny * nx:
            raise RuntimeError(f"{f}: expected {ny}x{nx} values, found {a.size}")
        out[name] = a.reshape(ny, nx)
    return out


def primitive_to_conserved(rho, u, v, p, gamma):
    """U = [rho, rho u, rho v, p/(gamma-1) + rho (u^2+v^2)/2] (src_WENO/fluid.cpp:86-93)."""
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)])


class Mesh:
    """The reference's ``Mesh``: grid parameters, primitive and conserved
    fields, ``bctype`` and (DG) the modal ``dof``, backed by a device Solver.

    ``Mesh(folder)`` reads a case directory; ``Mesh(ny, nx, da, gamma)`` makes
    a zero state.  Keyword options choose the method and precision.
    """

    def __init__(self, *args, method: str = "weno", order: int = 2, precision: str = "fp64",
                 limiter: str = "reference", flux: str = "hllc", boundary: str = "exchange",
                 device: int = 0, tvb_M: float = 50.0, recon: str = "weno5", tile_tpc: int = 0):
        self.method, self.order = method, int(order)
        self._opts = dict(method=method, order=order, precision=precision, limiter=limiter,
                          flux=flux, boundary=boundary, device=device, tvb_M=tvb_M, recon=recon,
                          tile_tpc=tile_tpc)
        self.nm = (self.order + 1) ** 2 if method == "dg" else 1
        if len(args) == 1:
            c = read_case(args[0])
            self.ny, self.nx, self.da, self.gamma = c["ny"], c["nx"], c["da"], c["gamma"]
            self.bctype = c["bctype"]
            self.rho, self.u, self.v, self.p = c["rho"], c["u"], c["v"], c["p"]
            U = primitive_to_conserved(self.rho, self.u, self.v, self.p, self.gamma)
        elif len(args) == 4:
            self.ny, self.nx, self.da, self.gamma = int(args[0]), int(args[1]), float(args[2]), float(args[3])
            self.bctype = np.zeros((self.ny, self.nx), np.int32)
            self.rho, self.u, self.v, self.p = (np.zeros((self.ny, self.nx)) for _ in range(4))
            U = np.zeros((4, self.ny, self.nx))
        else:
            raise TypeError("Mesh(folder) or Mesh(ny, nx, da, gamma)")
        self._host = np.zeros(self._shape()) if method == "dg" else U.copy()
        if method == "dg":
            self._host[:, 0] = U  # initDGModes, src_DG/fluid.cpp:173-182
        self._solver: Solver | None = None
        self._host_valid = True    # host copy current
        self._device_valid = False  # device copy current

    def _shape(self):
        return (4, self.nm, self.ny, self.nx) if self.method == "dg" else (4, self.ny, self.nx)

    # -- device sync -------------------------------------------------------------------
    def solver(self) -> Solver:
        """The device context, created and loaded on first use."""
        if self._solver is None:
            self._solver = Solver(**self._opts)
            self._solver.set_mesh(self.ny, self.nx, self.da, self.gamma, self.bctype)
        if not self._device_valid:
            self._solver.set_state(self._host)
            self._device_valid = True
        return self._solver

    def _pull(self):
        if not self._host_valid:
            self._host = self._solver.get_state()
            self._host_valid = True

    def _device_changed(self):
        self._host_valid = False

    def mark_host_modified(self) -> None:
        """Call after writing into the arrays returned by U0..U3 / dof."""
        self._pull()
        self._device_valid = False

    # -- reference field names ------------------------------------------------------------
    @property
    def state(self) -> np.ndarray:
        self._pull()
        return self._host

    @state.setter
    def state(self, value) -> None:
        v = np.ascontiguousarray(value, dtype=np.float64)
        if v.shape != self._shape():
            raise ValueError(f"state shape {v.shape} != {self._shape()}")
        self._host = v.copy()
        self._host_valid, self._device_valid = True, False

    def _cons(self, c):
        s = self.state
        return s[c, 0] if self.method == "dg" else s[c]

    U0 = property(lambda self: self._cons(0))
    U1 = property(lambda self: self._cons(1))
    U2 = property(lambda self: self._cons(2))
    U3 = property(lambda self: self._cons(3))

    @property
    def dof(self) -> np.ndarray:
        if self.method != "dg":
            raise AttributeError("dof exists for DG meshes only")
        return self.state

    def initDGModes(self) -> None:
        """Mode 0 = the cell values, higher modes zero (src_DG/fluid.cpp:173-182)."""
        s = self.state
        U = s[:, 0].copy()
        s[:] = 0.0
        s[:, 0] = U
        self._device_valid = False

    def syncCellAverages(self) -> None:
        """U0..U3 are views of mode 0 here, so there is nothing to copy
        (src_DG/fluid.cpp:190-196)."""

    def close(self) -> None:
        if self._solver is not None:
            self._pull()
            self._solver.close()
            self._solver = None
            self._device_valid = False


def computeRHS(mesh: Mesh, dt: float) -> np.ndarray:
    """computeRHS: fills ghosts of ``mesh`` in place and returns dU (WENO dU
    includes dt: src_WENO/fluid.cpp:454-460; DG dU = d(dof)/dt:
    src_DG/fluid.cpp:800-804)."""
    s = mesh.solver()
    dU = s.rhs(dt)
    mesh._device_changed()
    return dU


def updateMesh(mesh: Mesh, dt: float, rank: int = 0, num_procs: int = 1) -> None:
    """One SSP-RK3 step in place (src_WENO/fluid.cpp:468-493,
    src_DG/fluid.cpp:1005-1054).  With num_procs > 1, ``mesh`` is this rank's
    slab from splitMeshVertically and the step runs stage by stage with the
    exchange of its 3-column halos after every stage (and DG TVB pass) over the
    default torch.distributed group, whose ranks all call updateMesh."""
    if not 0 <= rank < num_procs:
        raise ValueError(f"rank {rank} outside 0..{num_procs - 1}")
    if num_procs == 1:
        mesh.solver().step(dt, 1)
    else:
        from . import slab
        s = mesh.solver()
        slab.slab_step([s], _slab_exchange(mesh, rank, num_procs), dt, 1)
        s.synchronize()
    mesh._device_changed()


def splitMeshVertically(original: Mesh, n: int) -> list[Mesh]:
    """splitMeshVertically (src_WENO/fluid.cpp:99-152, src_DG/fluid.cpp:249-312):
    n x-slab Meshes.  Slab k owns widths[k] = remain // (n - k) columns and has
    3 exchange columns (bctype -3) on every inner side, filled from the
    neighbour's columns; primitives, the conserved state (all DG modes) and
    bctype are copied.  Every slab needs at least 6 owned columns."""
    from . import slab
    prim = np.stack([original.rho, original.u, original.v, original.p])
    state_parts = slab.split_arrays(original.state, original.bctype, n)
    prim_parts = slab.split_arrays(prim, original.bctype, n)
    out = []
    for (st, b), (pr, _) in zip(state_parts, prim_parts):
        m = Mesh(original.ny, b.shape[1], original.da, original.gamma, **original._opts)
        m.bctype = b
        m.rho, m.u, m.v, m.p = (pr[c].copy() for c in range(4))
        m.state = st
        out.append(m)
    return out


def _slab_exchange(mesh: Mesh, rank: int, num_procs: int):
    from . import slab
    if not 0 <= rank < num_procs:
        raise ValueError(f"rank {rank} outside 0..{num_procs - 1}")
    ex = getattr(mesh, "_exchange", None)
    if ex is None or ex.solver is not mesh.solver() or (ex.rank, ex.nprocs) != (rank, num_procs):
        ex = slab.DistExchange(mesh.solver(), rank, num_procs)
        mesh._exchange = ex
    return ex


def exchangeConservativeColumns(mesh: Mesh, rank: int, num_procs: int) -> None:
    """exchangeConservativeColumns (src_WENO/fluid.cpp:192-198,
    src_DG/fluid.cpp:342-400): this rank's slab swaps the 3 columns next to
    each inner side, all variables and DG modes, with ranks rank-1 and rank+1
    of the default torch.distributed group."""
    if not 0 <= rank < num_procs:
        raise ValueError(f"rank {rank} outside 0..{num_procs - 1}")
    if num_procs == 1:
        return
    s = mesh.solver()
    _slab_exchange(mesh, rank, num_procs)(0)
    s.synchronize()
    mesh._device_changed()


def run(mesh: Mesh, dt: float, nsteps: int) -> None:
    """nsteps x updateMesh in one call (no host round trip between steps)."""
    mesh.solver().step(dt, nsteps)
    mesh._device_changed()


def applyLimiter(mesh: Mesh) -> None:
    """applyLimiter (src_DG/fluid.cpp:824-992), in place."""
    mesh.solver().limit()
    mesh._device_changed()


def computeMaxSpeed(mesh: Mesh, gamma: float | None = None) -> float:
    """WENO: computeMaxSpeed (src_WENO/fluid.cpp:539-553).  DG meshes use the
    DG rule of computeMaxSpeedDG_omp (src_DG/solver.cpp:26-64)."""
    if gamma is not None and float(gamma) != mesh.gamma:
        raise ValueError("gamma differs from the mesh's gamma")
    return mesh.solver().max_speed()


def recoverPrimitives(mesh: Mesh) -> None:
    """rho, u, v, p from the (cell-average) conserved state
    (src_WENO/fluid.cpp:500-515)."""
    prim = mesh.solver().recover_primitives()
    mesh.rho, mesh.u, mesh.v, mesh.p = prim[0], prim[1], prim[2], prim[3]


def dg_cfl_limit(order: int) -> float:
    """dgCFLLimit, src_DG/solver.cpp:15-17."""
    return 0.9 / (2.0 * (2 * order + 1))


def dg_safe_dt(lambda_max: float, h: float, order: int) -> float:
    """dgSafeDt, src_DG/solver.cpp:19-23."""
    return dg_cfl_limit(order) * h / max(lambda_max, 1e-7)


def saveMeshData(mesh: Mesh, rank: int, folder: str | os.PathLike) -> None:
    """Text snapshot U0_<rank>.dat..U3_<rank>.dat of the cell averages
    (src_WENO/fluid.cpp:558-577), 6 significant digits like the reference's
    default stream precision."""
    d = Path(folder) if folder else Path(".")
    d.mkdir(parents=True, exist_ok=True)
    for c, name in enumerate(("U0", "U1", "U2", "U3")):
        np.savetxt(d / f"{name}_{rank}.dat", mesh._cons(c), fmt="%.6g")


# ---- checkpoints and post-processing -------------------------------------------

def saveCheckpoint(mesh: Mesh, path: str | os.PathLike, t: float = 0.0, step: int = 0) -> Path:
    """Full-precision binary checkpoint of a Mesh: the whole conserved state
    (all DG modes, ghosts included, FP64 bit for bit), bctype, grid, gamma,
    the solver options, and the simulated time and step.  The reference only
    writes text snapshots of the cell averages (saveMeshData,
    src_WENO/fluid.cpp:558-577), from which a DG run cannot restart."""
    p = Path(path)
    if p.suffix != ".npz":
        p = p.with_suffix(".npz")
    np.savez(p, state=mesh.state, bctype=np.asarray(mesh.bctype, np.int32), grid=np.array([mesh.ny, mesh.nx]),
             da=mesh.da, gamma=mesh.gamma, t=t, step=step,
             options=np.array([f"{k}={v}" for k, v in mesh._opts.items()]))
    return p


def loadCheckpoint(path: str | os.PathLike, **overrides) -> tuple[Mesh, float, int]:
    """(mesh, t, step) from saveCheckpoint; keyword overrides replace saved
    options (e.g. precision="mixed" to continue a run on the fast path)."""
    z = np.load(Path(path), allow_pickle=False)
    opts = {}
    for item in z["options"]:
        k, v = str(item).split("=", 1)
        opts[k] = int(v) if k in ("order", "device", "tile_tpc") else float(v) if k == "tvb_M" else v
    opts.update(overrides)
    ny, nx = (int(x) for x in z["grid"])
    m = Mesh(ny, nx, float(z["da"]), float(z["gamma"]), **opts)
    m.bctype = z["bctype"].astype(np.int32)
    m.state = z["state"]
    return m, float(z["t"]), int(z["step"])


def computeMach(mesh: Mesh) -> tuple[np.ndarray, np.ndarray]:
    """(Mach, |u|) of the cell averages, the plot notebook's compute_mach
    (plot.ipynb cell 0), evaluated on the GPU from the device state."""
    import ctypes as C
    s = mesh.solver()
    mach = np.empty((mesh.ny, mesh.nx))
    speed = np.empty((mesh.ny, mesh.nx))
    N.check(N.lib().zk_mach_number(s._h, N.dptr(mach), N.dptr(speed)))
    return mach, speed


def combineRankSnapshots(folder: str | os.PathLike, n_ranks: int, ghost: int = 3) -> np.ndarray:
    """U[4][ny][nx] of a run the reference wrote as per-rank x-slabs
    (U<c>_<rank>.dat), with each slab's exchange columns dropped: the first
    slab keeps its left ring, the last its right ring (plot.ipynb
    load_and_combine_data)."""
    d = Path(folder)
    out = []
    for c in range(4):
        parts = []
        for r in range(n_ranks):
            a = np.loadtxt(d / f"U{c}_{r}.dat", ndmin=2)
            if n_ranks == 1:
                parts.append(a)
            elif r == 0:
                parts.append(a[:, :-ghost])
            elif r == n_ranks - 1:
                parts.append(a[:, ghost:])
            else:
                parts.append(a[:, ghost:-ghost])
        out.append(np.concatenate(parts, axis=1))
    return np.stack(out)
