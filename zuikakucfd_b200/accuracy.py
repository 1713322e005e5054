"""Accuracy study of the DG path on the periodic smooth wave (the DG P=2,
1024^2, TVB M=50, t=2 configuration): FP64 and mixed precision against the
exact translated solution and against each other.

    python -m zuikakucfd_b200.accuracy --n 1024 --order 2 --t-end 2 --limiter tvb
    python -m zuikakucfd_b200.accuracy --case jet --steps 2000      # the high-Mach jet

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
        precisions=("fp64", "mixed"), device: int = 0, chunk: int = 1000, v: float = 1.0) -> dict:
    """v = 1: the wave as configured (steady in the solvers' orientation);
    v = -1: translated along the diagonal, back in place at t = 2."""
    w = cases.smooth_wave(n, v=v)
    P = int(order)
    lam = math.sqrt(2.0) + math.sqrt(w.gamma * 1.0 / 0.8)
    dt0 = 0.9 / (2.0 * (2 * P + 1)) * w.da / lam
    steps = int(math.ceil(t_end / dt0))
    dt = t_end / steps
    d0 = cases.smooth_wave_modes(w, P) if init == "l2" else w.dg_state(P)
    ex = exact_cell_average(w, t_end)
    out = {"n": n, "order": P, "t_end": t_end, "steps": steps, "dt": dt, "limiter": limiter, "init": init,
           "velocity": [1.0, v], "paths": {}}
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


def restrict(a: np.ndarray, f: int) -> np.ndarray:
    """Interior (3-cell ring dropped) cell averages of a fine grid restricted
    to the grid f times coarser."""
    x = a[3:-3, 3:-3]
    n0, n1 = x.shape[0] // f, x.shape[1] // f
    return x.reshape(n0, f, n1, f).mean(axis=(1, 3))


def shock_refined_l1(order: int = 3, n: int = 64, refine: int = 4, t_end: float = 0.05, cfl_frac: float = 0.4,
                     seeds=(2, 3, 5, 7, 8, 9, 10), M: float = 50.0,
                     paths=(("fp64", "tvb"), ("mixed", "tvb"), ("mixed", "tvb_mlp")), device: int = 0) -> dict:
    """Density L1 error of DG paths on a seeded four-quadrant Riemann problem
    against a `refine` times finer FP64 + TVB solution of the same problem at
    the same physical time (cell averages restricted to the coarse grid).

    The state is the metric's four-quadrant case on the interior [0,1]^2 with
    the ring outside it (cases.four_quadrant(ring_outside=True)), so both grids
    hold the same physical problem.  dt = cfl_frac x the reference's DG CFL
    limit at the coarse grid, shortened so an integer number of steps reaches
    t_end; the fine run takes refine x the steps at dt / refine.  The first
    seed whose fine run stays clean (status word 0) is used.  Each coarse path
    is (precision, limiter); "tvb_mlp" runs the shipped learned indicator.
    Returns per path the L1 error (mean |rho - rho_fine|) and its ratio to the
    first path's, plus relative L1 / L-inf differences of each path's density
    and pressure against the first path."""
    P = int(order)

    def advance(case, dt, steps, prec, lim):
        with Solver(method="dg", order=P, precision=prec, limiter=lim, tvb_M=M, device=device) as s:
            s.set_mesh(case.ny, case.nx, case.da, case.gamma, case.bctype)
            if lim == "tvb_mlp":
                s.set_indicator()
            s.set_state(case.dg_state(P))
            left = steps
            while left:
                k = min(1000, left)
                s.step(dt, k)
                left -= k
            q = s.recover_primitives()
            return s.get_state(), q, s.status_word()

    t0 = time.perf_counter()
    for seed in seeds:
        cc = cases.four_quadrant(n, seed=seed, ring_outside=True)
        cf = cases.four_quadrant(n * refine, seed=seed, ring_outside=True)
        lam = cc.da / cases.cfl_dt(cc, 1.0)
        dt0 = cfl_frac * 0.9 / (2.0 * (2 * P + 1)) * cc.da / lam
        steps = int(math.ceil(t_end / dt0))
        dt = t_end / steps
        fine, _, st = advance(cf, dt / refine, steps * refine, "fp64", "tvb")
        if st == 0 and np.isfinite(fine[0, 0]).all():
            break
    else:
        raise RuntimeError("no seed gave a clean fine reference run")
    rho_ref = restrict(fine[0, 0], refine)
    out = {"order": P, "n": n, "refine": refine, "t_end": t_end, "steps": steps, "dt": dt, "seed": seed,
           "M": M, "reference": f"FP64 + TVB at {n * refine}^2", "paths": {}}
    base = None
    for prec, lim in paths:
        st, q, sw = advance(cc, dt, steps, prec, lim)
        rho = st[0, 0, 3:-3, 3:-3]
        key = f"{prec}+{lim}"
        rec = {"status_word": sw, "rho_l1_err": float(np.abs(rho - rho_ref).mean()),
               "rho_rel_l1_err": float(np.abs(rho - rho_ref).sum() / np.abs(rho_ref).sum())}
        prim = (q[0][3:-3, 3:-3], q[3][3:-3, 3:-3])
        if base is None:
            base = (key, rec["rho_l1_err"], prim)
        else:
            rec["rho_l1_err_ratio"] = rec["rho_l1_err"] / base[1]
            for name, a, b in (("density", prim[0], base[2][0]), ("pressure", prim[1], base[2][1])):
                d = np.abs(a - b)
                rec[f"rel_l1_{name}_vs_{base[0]}"] = float(d.sum() / np.abs(b).sum())
                rec[f"rel_linf_{name}_vs_{base[0]}"] = float(d.max() / np.abs(b).max())
        out["paths"][key] = rec
    out["seconds"] = time.perf_counter() - t0
    return out


def weno_refined_l1(n: int = 128, refine: int = 4, t_end: float = 0.05, cfl: float = 0.4, seed: int = 2,
                    device: int = 0) -> dict:
    """WENO5 FP64 and mixed paths on a seeded four-quadrant Riemann problem at
    n^2 against a `refine` times finer FP64 solution at the same physical time
    (cell averages restricted): density L1 errors, their ratio, and the mixed
    path's relative L1 / L-inf density and pressure differences from FP64.
    dt = cfl da / lambda0 (the reference driver's fixed-dt form), shortened so
    an integer number of steps reaches t_end."""
    t0 = time.perf_counter()
    cc = cases.four_quadrant(n, seed=seed, ring_outside=True)
    cf = cases.four_quadrant(n * refine, seed=seed, ring_outside=True)
    lam = cc.da / cases.cfl_dt(cc, 1.0)
    steps = int(math.ceil(t_end * lam / (cfl * cc.da)))
    dt = t_end / steps

    def advance(case, dt_, steps_, prec):
        with Solver(method="weno", precision=prec, device=device) as s:
            s.set_mesh(case.ny, case.nx, case.da, case.gamma, case.bctype)
            s.set_state(case.conserved())
            s.step(dt_, steps_)
            return s.get_state(), s.recover_primitives(), s.status_word()

    fine, _, stf = advance(cf, dt / refine, steps * refine, "fp64")
    rho_ref = restrict(fine[0], refine)
    out = {"method": "weno5", "n": n, "refine": refine, "t_end": t_end, "steps": steps, "dt": dt, "seed": seed,
           "reference": f"FP64 at {n * refine}^2", "reference_status_word": stf, "paths": {}}
    prims = {}
    for prec in ("fp64", "mixed"):
        st, q, sw = advance(cc, dt, steps, prec)
        rho = st[0, 3:-3, 3:-3]
        out["paths"][prec] = {"status_word": sw, "rho_l1_err": float(np.abs(rho - rho_ref).mean()),
                              "rho_rel_l1_err": float(np.abs(rho - rho_ref).sum() / np.abs(rho_ref).sum())}
        prims[prec] = (q[0][3:-3, 3:-3], q[3][3:-3, 3:-3])
    mx = out["paths"]["mixed"]
    mx["rho_l1_err_ratio"] = mx["rho_l1_err"] / out["paths"]["fp64"]["rho_l1_err"]
    for name, i in (("density", 0), ("pressure", 1)):
        d = np.abs(prims["mixed"][i] - prims["fp64"][i])
        mx[f"rel_l1_{name}_vs_fp64"] = float(d.sum() / np.abs(prims["fp64"][i]).sum())
        mx[f"rel_linf_{name}_vs_fp64"] = float(d.max() / np.abs(prims["fp64"][i]).max())
    out["seconds"] = time.perf_counter() - t0
    return out


def jet(nx: int = 2048, ny: int = 1024, steps: int = 2000, weno_cfl=(0.003, 0.01, 0.03), dg_cfl=(1.0,),
        precisions=("fp64", "mixed"), device: int = 0) -> dict:
    """The high-Mach jet (cases.high_mach_jet: rho = 5, u = 30 band, gamma =
    5/3, about Mach 80) advanced `steps` steps with WENO5 at each CFL number in
    weno_cfl (dt = cfl da / lambda0, the reference driver's fixed-dt form) and
    with DG P=1 at each dg_cfl x dgSafeDt (Persson + Zhang-Shu limiter), FP64 and
    mixed precision.  Per run: the device status word (1 NaN, 2 rho <= 0,
    4 p <= 0 seen), min density and pressure of the final cell averages, time;
    per method and CFL: mixed-vs-FP64 L1 / L-inf differences of rho and p."""
    c = cases.high_mach_jet(nx, ny)
    a_jet = math.sqrt(c.gamma * 0.4127 / 5.0)
    lam0 = 30.0 + a_jet
    runs = []
    for method, order, cfls in (("weno", 2, weno_cfl), ("dg", 1, tuple(dg_cfl))):
        for cfl in cfls:
            dt = cfl * c.da / lam0 if method == "weno" else cfl * 0.9 / (2.0 * 3.0) * c.da / lam0
            res, prim = {}, {}
            for prec in precisions:
                with Solver(method=method, order=order, precision=prec, device=device) as s:
                    s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
                    s.set_state(c.conserved() if method == "weno" else c.dg_state(order))
                    t0 = time.perf_counter()
                    s.step(dt, steps)
                    s.synchronize()
                    secs = time.perf_counter() - t0
                    q = s.recover_primitives()
                    st = s.status_word()
                rho, p = q[0][3:-3, 3:-3], q[3][3:-3, 3:-3]
                fin = bool(np.isfinite(rho).all() and np.isfinite(p).all())
                prim[prec] = (rho, p)
                res[prec] = {"status_word": st, "finite": fin, "seconds": secs,
                             "rho_min": float(np.nanmin(rho)), "p_min": float(np.nanmin(p))}
            row = {"method": method, "order": order if method == "dg" else None, "cfl": cfl, "dt": dt,
                   "steps": steps, "paths": res}
            if len(prim) == 2 and all(v["finite"] for v in res.values()):
                (r64, p64), (rmx, pmx) = prim["fp64"], prim["mixed"]
                row["mixed_vs_fp64"] = {
                    "rho_l1_rel": float(np.abs(rmx - r64).sum() / np.abs(r64).sum()),
                    "rho_linf": float(np.abs(rmx - r64).max()),
                    "p_l1_rel": float(np.abs(pmx - p64).sum() / np.abs(p64).sum()),
                    "p_linf": float(np.abs(pmx - p64).max())}
            runs.append(row)
    return {"case": f"high-Mach jet {nx}x{ny}", "runs": runs}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--order", type=int, default=2)
    ap.add_argument("--t-end", type=float, default=2.0)
    ap.add_argument("--limiter", default="tvb")
    ap.add_argument("--init", default="l2", choices=["l2", "reference"])
    ap.add_argument("--precisions", default="fp64,mixed")
    ap.add_argument("--case", default="wave", choices=["wave", "jet"])
    ap.add_argument("--steps", type=int, default=2000, help="jet: steps per run")
    ap.add_argument("--v", type=float, default=1.0, help="wave: row-direction velocity (-1: translating)")
    ap.add_argument("--dg-cfl", default="1.0", help="jet: comma-separated multiples of dgSafeDt for DG P=1")
    a = ap.parse_args(argv)
    if a.case == "jet":
        print(json.dumps(jet(steps=a.steps, precisions=a.precisions.split(","),
                             dg_cfl=tuple(float(x) for x in a.dg_cfl.split(",")))), flush=True)
        return 0
    print(json.dumps(run(a.n, a.order, a.t_end, a.limiter, a.init, a.precisions.split(","), v=a.v)), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
