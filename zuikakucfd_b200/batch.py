"""Batched runner over the C ABI (zk_batch_*): many independent problems of
uneven grid sizes, WENO and DG mixed, advanced together on one GPU.

    with Batch(policy="sjf") as b:
        for spec in batch_problems(256, seed=0):
            b.add(**spec)
        report = b.run()           # aggregate cell/DOF updates, latency p50/p99
        rho = b.get_state(0)[0]

The reference advances one mesh per process (src_WENO/solver.cpp:159-190,
src_DG/solver.cpp:270-310); a batch keeps each problem's own CFL time step,
step count and boundary handling and advances all of them with persistent
kernels (one launch per RK stage and problem group) replayed from a CUDA graph.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from . import cases


class Batch:
    def __init__(self, policy: str = "all", active_cells: float = 8e6, graph_steps: int = 10,
                 autotune: int = 1, arena_bytes: int = 0, device: int = 0, weno_variant: int = -1,
                 dg_variant: int = -1):
        L = N.lib()
        o = N.zk_batch_options()
        L.zk_batch_default_options(C.byref(o))
        o.device = int(device)
        o.policy = N.POLICY[policy]
        o.active_cells = float(active_cells)
        o.graph_steps = int(graph_steps)
        o.autotune = int(autotune)
        o.arena_bytes = int(arena_bytes)
        o.weno_variant = int(weno_variant)
        o.dg_variant = int(dg_variant)
        h = C.c_void_p()
        N.check(L.zk_batch_create(C.byref(o), C.byref(h)))
        self._h = h
        self.device = int(device)
        self._shapes: list[tuple] = []
        self._steps: list[int] = []

    # -- lifetime ----------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().zk_batch_destroy(self._h)
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

    # -- problems ------------------------------------------------------------------
    def add(self, bctype, da: float, gamma: float, state, nsteps: int, cfl: float, method: str = "weno",
            order: int = 2, precision: str = "fp64", limiter: str = "reference", flux: str = "hllc",
            boundary: str = "exchange") -> int:
        """Register one problem; state is U[4][ny][nx] (WENO) or
        dof[4][NM][ny][nx] (DG).  Returns its id."""
        b = np.ascontiguousarray(bctype, dtype=np.int32)
        ny, nx = b.shape
        nm = (int(order) + 1) ** 2 if method == "dg" else 1
        shape = (4, nm, ny, nx) if method == "dg" else (4, ny, nx)
        s = np.ascontiguousarray(state, dtype=np.float64)
        if s.shape != shape:
            raise ValueError(f"state shape {s.shape} != {shape}")
        o = N.zk_options()
        N.lib().zk_default_options(C.byref(o))
        o.method = N.METHOD[method]
        o.order = int(order)
        o.precision = N.PRECISION[precision]
        o.limiter = N.LIMITER[limiter]
        o.flux = N.FLUX[flux]
        o.boundary = N.BOUNDARY[boundary]
        o.device = self.device
        pid = C.c_int()
        N.check(N.lib().zk_batch_add(self._h, C.byref(o), ny, nx, float(da), float(gamma),
                                     b.ctypes.data_as(C.POINTER(C.c_int32)), N.dptr(s), int(nsteps),
                                     float(cfl), C.byref(pid)))
        self._shapes.append(shape)
        self._steps.append(int(nsteps))
        return pid.value

    def run(self) -> dict:
        r = N.zk_batch_report()
        N.check(N.lib().zk_batch_run(self._h, C.byref(r)))
        return {f: getattr(r, f) for f, _ in r._fields_}

    # -- results ---------------------------------------------------------------------
    def get_state(self, pid: int) -> np.ndarray:
        out = np.empty(self._shapes[pid])
        N.check(N.lib().zk_batch_get_state(self._h, int(pid), N.dptr(out)))
        return out

    def info(self, pid: int) -> dict:
        p = N.zk_batch_problem()
        N.check(N.lib().zk_batch_problem_info(self._h, int(pid), C.byref(p)))
        d = {f: getattr(p, f) for f, _ in p._fields_}
        d["state"] = N.BATCH_STATE[d["state"]]
        return d

    def dt_history(self, pid: int, n: int | None = None) -> np.ndarray:
        n = self._steps[pid] if n is None else int(n)
        out = np.empty(n)
        N.check(N.lib().zk_batch_dt_history(self._h, int(pid), N.dptr(out), n))
        return out

    def groups(self) -> list[dict]:
        """Per problem group: method, precision, order, the tile the autotuner
        chose for its stage kernel (cells per tile, threads per tile and per
        cell) and its CTAs per SM."""
        L = N.lib()
        ng = C.c_int()
        N.check(L.zk_batch_group_config(self._h, -1, None, None, None, None, None, C.byref(ng)))
        out = []
        inv_m = {v: k for k, v in N.METHOD.items()}
        inv_p = {v: k for k, v in N.PRECISION.items()}
        for g in range(ng.value):
            v = [C.c_int() for _ in range(5)]
            N.check(L.zk_batch_group_config(self._h, g, *[C.byref(x) for x in v], None))
            m, p, o, var, ctas = (x.value for x in v)
            t = [C.c_int() for _ in range(3)]
            N.check(L.zk_batch_group_tile(self._h, g, *[C.byref(x) for x in t]))
            rows, cols, threads = (x.value for x in t)
            out.append({"method": inv_m[m], "precision": inv_p[p], "order": o, "variant": var,
                        "tile_rows": rows, "tile_cols": cols, "threads_per_tile": threads,
                        "threads_per_cell": threads / (rows * cols), "ctas_per_sm": ctas})
        return out


def batch_sides(n: int = 256, seed: int = 0, sides=range(128, 1025, 128)) -> list[int]:
    """Side lengths of the batched-serving workload's problems (uniform draw)."""
    sides = list(sides)
    drawn = np.random.default_rng(seed).integers(0, len(sides), size=n)
    return [int(sides[k]) for k in drawn]


def batch_problems(n: int = 256, seed: int = 0, sides=range(128, 1025, 128), nsteps: int = 500,
                   precision: str = "mixed", weno_cfl: float = 0.4, dg_cfl: float = 0.5,
                   dg_order: int = 2):
    """The batched-serving workload: n seeded four-quadrant problems (the
    cases.four_quadrant generator), side lengths drawn uniformly from `sides`,
    the first half WENO5, the second half DG P=dg_order; each runs nsteps
    steps at its own CFL time step.  Yields keyword arguments of Batch.add."""
    for i, side in enumerate(batch_sides(n, seed, sides)):
        c = cases.four_quadrant(side, seed=int(seed) * 100003 + i)
        if i < n // 2:
            yield dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.conserved(), nsteps=nsteps,
                       cfl=weno_cfl, method="weno", precision=precision)
        else:
            yield dict(bctype=c.bctype, da=c.da, gamma=c.gamma, state=c.dg_state(dg_order), nsteps=nsteps,
                       cfl=dg_cfl, method="dg", order=dg_order, precision=precision)
