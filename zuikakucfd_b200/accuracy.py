"""Accuracy study of the DG path on the periodic smooth wave (the DG P=2,
1024^2, TVB M=50, t=2 configuration): FP64 and mixed precision against the
exact translated solution and against each other.

    python -m zuikakucfd_b200.accuracy --n 1024 --order 2 --t-end 2 --limiter tvb

rho = 1 + 0.2 sin(pi (x + y)), u = v = p = 1 on [0,2]^2, periodic; the exact
solution is rho0(x - t, y + t) (cases.smooth_wave_exact: the solvers' v points
along increasing row index, downwards), and at t = 2 it is the initial field
in either orientation.  The initial state is the L2 projection onto the DG basis
(cases.smooth_wave_modes; --init reference uses the reference's cell-centre
mode-0 start instead).  dt = 0.9 / (2 (2P+1)) h / lambda, lambda = max |u| + a
= sqrt(2) + sqrt(gamma p / rho_min), the reference's dgSafeDt at its CFL limit,
shortened so that an integer number of steps reaches t_end.  Prints one JSON
object: L1 (mean absolute) and L-inf errors of the cell-average density and
pressure against the exact cell averages, and of the mixed path against FP64.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import cases
from .fluid import Solver


def exact_cell_average(case: cases.Case, t: float, amplitude: float = 0.2) -> np.ndarray:
    """Interior cell averages of rho at time t (sin averages by sinc^2 over a square)."""
    kh = math.pi * case.da / 2.0
    return 1.0 + (cases.smooth_wave_exact(case, t, amplitude) - 1.0) * (math.sin(kh) / kh) ** 2


def run(n: int = 1024, order: int = 2, t_end: float = 2.0, limiter: str = "tvb", init: str = "l2",
        precisions=("fp64", "mixed"), device: int = 0, chunk: int = 1000) -> dict:
    w = cases.smooth_wave(n)
    P = int(order)
    lam = math.sqrt(2.0) + math.sqrt(w.gamma * 1.0 / 0.8)
    dt0 = 0.9 / (2.0 * (2 * P + 1)) * w.da / lam
    steps = int(math.ceil(t_end / dt0))
    dt = t_end / steps
    d0 = cases.smooth_wave_modes(w, P) if init == "l2" else w.dg_state(P)
    ex = exact_cell_average(w, t_end)
    out = {"n": n, "order": P, "t_end": t_end, "steps": steps, "dt": dt, "limiter": limiter, "init": init,
           "paths": {}}
    states = {}
    for prec in precisions:
        with Solver(method="dg", order=P, precision=prec, limiter=limiter, boundary="periodic",
                    device=device) as s:
            s.set_mesh(w.ny, w.nx, w.da, w.gamma, w.bctype)
            s.set_state(d0)
            t0 = time.perf_counter()
            left = steps
            while left:
                k = min(chunk, left)
                s.step(dt, k)
                left -= k
            s.synchronize()
            secs = time.perf_counter() - t0
            prim = s.recover_primitives()
            status = s.status_word()
        rho, p = prim[0][3:-3, 3:-3], prim[3][3:-3, 3:-3]
        states[prec] = (rho, p)
        out["paths"][prec] = {
            "seconds": secs, "status_word": status,
            "rho_l1": float(np.abs(rho - ex).mean()), "rho_linf": float(np.abs(rho - ex).max()),
            "p_l1": float(np.abs(p - 1.0).mean()), "p_linf": float(np.abs(p - 1.0).max()),
            "dof_updates_per_s": (n * n) * 4 * (P + 1) ** 2 * steps / secs}
    if "fp64" in states and "mixed" in states:
        (r64, p64), (rmx, pmx) = states["fp64"], states["mixed"]
        out["mixed_vs_fp64"] = {
            "rho_l1": float(np.abs(rmx - r64).mean()), "rho_linf": float(np.abs(rmx - r64).max()),
            "p_l1": float(np.abs(pmx - p64).mean()), "p_linf": float(np.abs(pmx - p64).max()),
            "rho_l1_error_ratio": out["paths"]["mixed"]["rho_l1"] / out["paths"]["fp64"]["rho_l1"]}
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--order", type=int, default=2)
    ap.add_argument("--t-end", type=float, default=2.0)
    ap.add_argument("--limiter", default="tvb")
    ap.add_argument("--init", default="l2", choices=["l2", "reference"])
    ap.add_argument("--precisions", default="fp64,mixed")
    a = ap.parse_args(argv)
    print(json.dumps(run(a.n, a.order, a.t_end, a.limiter, a.init, a.precisions.split(","))), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
