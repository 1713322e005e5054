#!/usr/bin/env python
"""DOF-updates/s of the ZuikakuCFD per-step compute on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--no-cpu-baseline]

One "step" is one SSP-RK3 step (updateMesh) over the whole grid of the
workload, inputs resident in HBM.  value = DOF-updates/s of the whole job
(cell updates x DOFs per cell, summed over ranks; each rank owns an
independent seeded problem: weak scaling, no data-path collective).  rank 0
prints one JSON line.  Timing: CUDA events on the library's stream around
exactly K steps, barrier + synchronize on both sides, max over ranks.

--impl reference times the reference's own CPU implementation (its sources
built unmodified as oracle/_ref, x-slab threads standing in for MPI ranks) on
a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DOF-updates/s on 1 B200: mixed-prec+learned limiter vs plain FP64 at equal L1"
UNIT = "DOF-updates/s"

# Algorithmic work per updated cell per RK stage (face-deduplicated, 1 flop per
# add/sub/mul/div/sqrt/min/max): WENO5 = 2 faces x (8 one-sided
# reconstructions x 66 + HLLC 117) + flux difference 24 + RK combine 12.
WENO_FLOPS_PER_CELL_STAGE = 1330.0


# DG: volume NQ^2 (28 NM + 40) + faces 2 NQ (32 NM + 127) + inverse mass 4 NM
# + RK combine 16 NM, rounded (NM = (P+1)^2 modes, NQ = P+1 points).
FLOPS_PER_CELL_STAGE = {("weno", 0): WENO_FLOPS_PER_CELL_STAGE, ("dg", 1): 1700.0, ("dg", 2): 5300.0,
                        ("dg", 3): 13200.0}


# DRAM bytes per launch of the dominant kernel, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of a 512^2 instance of the
# workload (256,036 updated cells), scaled to a full launch by the updated
# cells; None where not captured.  Keyed by (workload, precision):
# (bytes per updated cell, what was captured).
KERNEL_TRAFFIC_PER_CELL: dict = {
    ("dg3_fq_2048", "mixed", "dg_stage_mixed_pair_kernel"): (
        977.2, "dg_stage_mixed_pair_kernel<3,float,float,MLP> (stage 2) at 512^2: 201.8 MB read + 48.3 MB written"),
    ("weno_fq_2048", "mixed", "weno_stage_mixed_kernel"): (
        57.7, "weno_stage_mixed_kernel (stage 1) at 2048^2: 139.2 MB read + 101.4 MB written"),
}
# the mixed DG stage kernel for each threads-per-cell choice of the tuner
DG_MIXED_KERNEL = {1: "dg_stage_mixed_kernel", 2: "dg_stage_mixed_pair_kernel", 4: "dg_stage_mixed_quad_kernel"}


def make_workload(name: str, rank: int):
    from zuikakucfd_b200 import cases
    seed = 1000 + rank
    if name == "weno_jet_2048x1024":
        c = cases.high_mach_jet(2048, 1024)
        dt = 0.003 * c.da / (30.0 + float(np.sqrt(c.gamma * 0.4127 / 5.0)))
        return dict(case=c, method="weno", order=0, dof_per_cell=4, dt=dt, opts={},
                    desc="high-Mach jet 2048x1024 (rho=5,u=30 band, gamma=5/3), WENO5+HLLC+SSP-RK3, CFL 0.003")
    if name.startswith("weno_fq_"):
        n = int(name.split("_")[-1])
        c = cases.four_quadrant(n, seed=seed)
        return dict(case=c, method="weno", order=0, dof_per_cell=4, dt=cases.cfl_dt(c, 0.4), opts={},
                    desc=f"seeded four-quadrant Riemann {n}x{n} (seed {seed}), WENO5+HLLC+SSP-RK3, CFL 0.4")
    if name.startswith("dg") and "_fq_" in name:
        P = int(name[2])
        n = int(name.split("_")[-1])
        c = cases.four_quadrant(n, seed=seed)
        lam = c.da / cases.cfl_dt(c, 1.0)
        dt = 0.5 * 0.9 / (2.0 * (2 * P + 1)) * c.da / lam
        learned = P == 3
        return dict(case=c, method="dg", order=P, dof_per_cell=4 * (P + 1) ** 2, dt=dt,
                    opts={"fp64": {"limiter": "tvb"}, "mixed": {"limiter": "tvb_mlp" if learned else "tvb"}},
                    desc=f"seeded four-quadrant Riemann {n}x{n} (seed {seed}), DG P={P} HLLC SSP-RK3, "
                         + ("mixed precision + learned troubled-cell indicator gating TVB (M=50) limiting vs "
                            "plain FP64 + TVB limiting" if learned else "TVB limiter M=50")
                         + ", half the reference's CFL limit")
    if name.startswith("dg") and "_wave_" in name:
        P = int(name[2])
        n = int(name.split("_")[-1])
        c = cases.smooth_wave(n)
        dt = 0.9 / (2.0 * (2 * P + 1)) * c.da / 2.74
        return dict(case=c, method="dg", order=P, dof_per_cell=4 * (P + 1) ** 2, dt=dt,
                    opts={"limiter": "tvb", "boundary": "periodic"},
                    desc=f"periodic smooth wave {n}^2 on [0,2]^2, DG P={P} HLLC SSP-RK3, dt at the reference's CFL limit")
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """SM clock and throttle reasons sampled during the timed region: NVML
    polled every ~2 ms from a thread (the timed call releases the GIL)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device: int):
        self.device = device
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.device]) if vis else self.device
            self.h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.nv = nv
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
        return self

    def _poll(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((float(mhz), int(r)))
            except Exception:
                pass
            time.sleep(0.002)

    def __exit__(self, *exc):
        self._stop.set()
        if self.nv is not None:
            self.t.join(timeout=2)

    def summary(self) -> dict:
        sm = [m for m, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(sm), "source": "NVML, polled every 2 ms"}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def allreduce_max(pg, x: float) -> float:
    """Max over ranks (the slowest rank's time); a device tensor under NCCL,
    a host tensor under gloo."""
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def measure_peaks(device: int) -> dict:
    import ctypes as C
    from zuikakucfd_b200 import _native as N
    out = {}
    for kind, name in ((0, "fp64_tflops"), (1, "fp32_tflops")):
        v = C.c_double()
        N.check(N.lib().zk_peak_flops(device, kind, C.byref(v)))
        out[name] = v.value
    return out


def _ref_state(w):
    c = w["case"]
    return c.conserved() if w["method"] == "weno" else c.dg_state(w["order"])


def _ref_slabs(R, w, state, bct, nsteps, cores):
    """(ms of the slowest slab, updated cells) for the reference's own
    updateMesh run on `cores` x-slabs (threads standing in for MPI ranks)."""
    c = w["case"]
    if w["method"] == "weno":
        return R.weno_slabs_timed(state, bct, c.da, c.gamma, w["dt"], nsteps, cores)
    return R.dg_slabs_timed(w["order"], state, bct, c.da, c.gamma, w["dt"], nsteps, cores)


def _ref_strip(R, w, cores, target_ms):
    """A horizontal strip of the workload's grid sized so that one reference
    step takes about target_ms on this host (bounded CPU sample)."""
    c = w["case"]
    full = _ref_state(w)
    probe = min(c.ny, 64)
    st = np.ascontiguousarray(full[..., :probe, :])
    b = np.ascontiguousarray(c.bctype[:probe]).copy()
    b[-3:] = -1
    ms, _ = _ref_slabs(R, w, st, b, 1, cores)
    rows = int(min(c.ny, max(16, probe * target_ms / max(ms, 1e-3))))
    st = np.ascontiguousarray(full[..., :rows, :])
    b = np.ascontiguousarray(c.bctype[:rows]).copy()
    if rows < c.ny:
        b[-3:] = -1
    return st, b, rows


def cpu_baseline(w: dict, seconds: float = 15.0) -> dict:
    """The reference's own sources (oracle/_ref, Makefile flags) on this host's
    cores: x-slab threads standing in for MPI ranks, a bounded sample."""
    from oracle.oracle import Reference, reference_available
    if not reference_available("faithful"):
        return {"value": None, "unavailable": "oracle/_ref not built"}
    c = w["case"]
    cores = max(1, min(os.cpu_count() or 1, 64))
    R = Reference("faithful")
    st, b, rows = _ref_strip(R, w, cores, 2000.0)
    ms, cells = _ref_slabs(R, w, st, b, 1, cores)
    n = max(1, int(seconds * 1e3 / max(ms, 1.0)))
    ms, cells = _ref_slabs(R, w, st, b, n, cores)
    v = cells * w["dof_per_cell"] * n / (ms * 1e-3)
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{n} x updateMesh on a {rows}x{c.nx} strip of the {c.ny}x{c.nx} grid split into "
                      f"{cores} x-slabs (one thread per slab, reference Makefile flags at ISA {R.isa}, "
                      "halo exchange omitted)",
            "ms": ms}


def run_reference_arm(args, w) -> dict:
    from oracle.oracle import Reference, reference_available
    if not reference_available("faithful"):
        return {"impl": "reference", "unavailable": "oracle/_ref (reference built from its sources) missing"}
    c = w["case"]
    cores = max(1, min(os.cpu_count() or 1, 64))
    R = Reference("faithful")
    st, b, rows = _ref_strip(R, w, cores, 1500.0)
    for _ in range(args.warmup):
        _ref_slabs(R, w, st, b, 1, cores)
    ms, cells = _ref_slabs(R, w, st, b, args.steps, cores)
    v = cells * w["dof_per_cell"] * args.steps / (ms * 1e-3)
    sample = (f"{rows}x{c.nx} strip of the {c.ny}x{c.nx} grid per step, {cores} x-slab threads, "
              f"reference Makefile flags at ISA {R.isa}")
    return {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": args.workload, "grid": [c.ny, c.nx]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_e2e(s, w, U0, args, world, dofs, pg) -> dict:
    """End to end through the public C ABI with host buffers: the reference
    driver's loop -- computeMaxSpeed -> dt on the host -> updateMesh -- with
    the state uploaded from pinned host memory at the start and read back at
    the end, all inside the timed region.  The WENO driver takes the max wave
    speed every step (src_WENO/solver.cpp:159-178), the DG driver every 10
    steps (cfl_recheck_interval, src_DG/solver.cpp:267-289).  At least 100
    steps per upload (a run of the reference does thousands), K if larger."""
    import ctypes as C
    import torch
    from zuikakucfd_b200 import _native as N
    host_in = torch.from_numpy(np.ascontiguousarray(U0)).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    state_bytes = host_in.numel() * 8
    every = 10 if w["method"] == "dg" else 1
    steps = max(args.steps, 100)
    steps = -(-steps // every) * every
    L = N.lib()
    lam = C.c_double()
    barrier(pg)
    t0 = time.perf_counter()
    N.check(L.zk_set_state(s._h, C.cast(host_in.data_ptr(), C.POINTER(C.c_double))))
    for _ in range(steps // every):
        N.check(L.zk_max_speed(s._h, C.byref(lam)))
        N.check(L.zk_step(s._h, C.c_double(w["dt"]), every))
    N.check(L.zk_get_state(s._h, C.cast(host_out.data_ptr(), C.POINTER(C.c_double))))
    e2e_s = allreduce_max(pg, time.perf_counter() - t0)
    return {"value": world * dofs * steps / e2e_s, "unit": UNIT,
            "h2d_bytes_per_step": state_bytes / steps,
            "d2h_bytes_per_step": state_bytes / steps + 8.0 / every,
            "steps": steps,
            "what": f"the reference driver's loop: zk_max_speed (8 B read back) every {every} step(s), then "
                    f"zk_step(dt, {every}); state H2D from pinned host at the start, D2H at the end, "
                    f"{steps} steps, amortised per step; host wall clock"}


def measure_single(name: str, args, rank: int, world: int, local: int, pg, e2e: bool = True,
                   cpu_seconds: float = 15.0, refined: bool = True) -> dict | None:
    """One single-problem workload: the plain FP64 path (the metric's
    baseline), then the mixed path (the headline), each timed over exactly K
    steps after W warm-up steps.  rank 0 returns the line's fields, the other
    ranks None."""
    w = make_workload(name, rank)
    c = w["case"]
    U0 = c.conserved() if w["method"] == "weno" else c.dg_state(w["order"])
    cells = c.fluid_cells
    dofs = cells * w["dof_per_cell"]

    # fp64: the reference-arithmetic path (--fmad=false, bit-exact against the
    # reference built without contraction); fp64_fma: the same kernels with
    # fused multiply-adds (the fastest plain-FP64 path); mixed: the headline
    paths = {}
    for prec in (["fp64", "fp64_fma", "mixed"] if not args.fp64_only else ["fp64"]):
        s = open_solver(w, c, U0, prec, local)
        for _ in range(args.warmup):
            s.step(w["dt"], 1)
        s.synchronize()
        barrier(pg)
        with ClockSampler(local) as clk:
            ms = s.step_timed(w["dt"], args.steps)  # CUDA events on the library stream
            s.synchronize()
        barrier(pg)
        ms_max = allreduce_max(pg, ms)
        paths[prec] = {"ms": ms, "ms_max": ms_max, "status": s.status_word(), "clocks": clk.summary(),
                       "value": world * dofs * args.steps / (ms_max * 1e-3), "solver": s,
                       "tpc": s.tile_tpc() if (w["method"] == "dg" and prec == "mixed") else None}
    head = "mixed" if "mixed" in paths else "fp64"
    hp = paths[head]
    # equal-L1 diagnostics: (a) both paths advanced the same steps from the
    # same state: relative L1 and Linf differences of the cell-average density
    # and pressure (primitives recovered in FP64); (b) below, each path's L1
    # error against a 4x finer FP64 solution of the same problem
    eq = None
    if "mixed" in paths:
        q64 = paths["fp64"]["solver"].recover_primitives()
        qmx = paths["mixed"]["solver"].recover_primitives()
        eq = {"steps_compared": args.warmup + args.steps}
        for nm, f in (("density", 0), ("pressure", 3)):
            d = np.abs(qmx[f] - q64[f])
            eq[f"rel_l1_{nm}_mixed_vs_fp64"] = float(d.sum() / np.abs(q64[f]).sum())
            eq[f"rel_linf_{nm}_mixed_vs_fp64"] = float(d.max() / np.abs(q64[f]).max())

    e2e_rec = run_e2e(hp["solver"], w, U0, args, world, dofs, pg) if e2e else None
    for pth in paths.values():
        pth["solver"].close()
    if rank != 0:
        return None

    if eq is not None and refined:
        eq["refined"] = refined_l1(w)
        pr = eq["refined"]["paths"]
        base = next(iter(pr))
        mixed_key = [k for k in pr if k.startswith("mixed")][-1]
        eq["rel_l1_err_fp64"] = pr[base]["rho_rel_l1_err"]
        eq["rel_l1_err_mixed"] = pr[mixed_key]["rho_rel_l1_err"]
        eq["l1_err_ratio_mixed_over_fp64"] = pr[mixed_key]["rho_l1_err_ratio"]
        eq["equal_l1_met"] = bool(pr[mixed_key]["rho_l1_err_ratio"] <= 1.1)
    peaks = measure_peaks(local)
    peaks_file = ROOT / "MEASURED_PEAKS.json"
    hbm_peak = json.loads(peaks_file.read_text())["hbm_gbs"] if peaks_file.exists() else 6650.0
    roofs = {}
    fl = FLOPS_PER_CELL_STAGE[(w["method"], w["order"])]
    nvar = w["dof_per_cell"]
    for prec, pth in paths.items():
        stage_ms = pth["ms"] / (3 * args.steps)  # time of one RK stage (all its launches)
        achieved = cells * fl / (stage_ms * 1e-3) / 1e12
        f64 = prec != "mixed"
        pk = peaks["fp64_tflops"] if f64 else peaks["fp32_tflops"]
        # minimal traffic per stage: stage input + U^n + output (+ kind byte)
        bpv = 8.0 if (f64 or w["method"] == "weno") else 4.0
        hbm_bytes = cells * (nvar * (bpv + 8.0 + bpv) + 1.0)
        if w["method"] == "weno":
            kname = "weno_stage_fp64_kernel" if f64 else "weno_stage_mixed_kernel"
        else:
            # the mixed stage kernel the context's tuner chose (threads per cell)
            kname = ("dg_face_kernel x2 + dg_cell_kernel (one stage)" if f64
                     else DG_MIXED_KERNEL.get(pth["tpc"], "dg_stage_mixed_kernel"))
        if prec == "fp64_fma":
            kname = ("weno_stage_fp64_kernel, FMA-contracted build" if w["method"] == "weno"
                     else "dg_stage_fused_fp64_kernel (one fused FP64 launch per stage, FMA)")
        roofs[prec] = {
            "bound": "fp64" if f64 else "fp32", "achieved": achieved, "peak": pk,
            "unit": "TFLOP/s", "frac": achieved / pk,
            "traffic": (KERNEL_TRAFFIC_PER_CELL[(name, prec, kname)][0] * cells
                        if (name, prec, kname) in KERNEL_TRAFFIC_PER_CELL else None),
            "traffic_source": (KERNEL_TRAFFIC_PER_CELL[(name, prec, kname)][1] + ", scaled by updated cells"
                               if (name, prec, kname) in KERNEL_TRAFFIC_PER_CELL else None),
            "algorithmic_bytes": hbm_bytes,
            "kernel": kname, "threads_per_cell": pth["tpc"], "flops_per_cell_stage": fl,
            "avg_launch_ms": stage_ms,
            "peak_source": "measured: zk_peak_flops FMA microbenchmark on this GPU "
                           "(MEASURED_PEAKS.json has no FP64/FP32 figure)",
            "hbm": {"achieved_gbs": hbm_bytes / (stage_ms * 1e-3) / 1e9, "peak_gbs": hbm_peak,
                    "frac": hbm_bytes / (stage_ms * 1e-3) / 1e9 / hbm_peak}}
    cpu = ({"value": None, "skipped": True} if args.no_cpu_baseline or world > 1
           else cpu_baseline(w, cpu_seconds))
    return {"metric": METRIC, "value": hp["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": hp["ms_max"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if head == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": name, "desc": w["desc"], "grid": [c.ny, c.nx],
                       "updated_cells": cells, "dof_per_cell": w["dof_per_cell"], "precision": head,
                       "l2": "working set (3 FP64 states = %.0f MB) larger than the 126 MB L2" %
                             (3 * U0.nbytes / 1e6),
                       "parallelism": f"replicas x{world} (independent seeded problems)"},
            "fp64_value": paths["fp64"]["value"], "fp64_fma_value": paths.get("fp64_fma", {}).get("value"),
            "equal_l1": eq,
            "cell_updates_per_s": hp["value"] / w["dof_per_cell"],
            "speedup_vs_fp64": hp["value"] / paths["fp64"]["value"],
            "speedup_vs_best_fp64": hp["value"] / max(v["value"] for k, v in paths.items() if k != "mixed"),
            "clocks": hp["clocks"], "e2e": e2e_rec,
            "gpu_launches": gpu_launches(w, head) * args.steps,
            "roofline": roofs[head], "roofline_fp64": roofs["fp64"], "roofline_fp64_fma": roofs.get("fp64_fma"),
            "cpu_baseline": cpu,
            "status_word": {p: v["status"] for p, v in paths.items()}, "peaks": peaks}


def refined_l1(w: dict) -> dict:
    """Density L1 error of the workload's FP64 and mixed paths on a 128^2
    instance of its four-quadrant problem against a 4x finer FP64 solution
    (512^2) at t = 0.05: the 'at equal L1' of the metric, checked rather than
    inferred.  DG: FP64 + TVB, mixed + TVB and (P=3) mixed + learned
    indicator; WENO5: FP64 and mixed."""
    from zuikakucfd_b200 import accuracy
    if w["method"] == "dg":
        P = w["order"]
        paths = (("fp64", "tvb"), ("mixed", "tvb")) + ((("mixed", "tvb_mlp"),) if P == 3 else ())
        return accuracy.shock_refined_l1(order=P, n=128, refine=4, t_end=0.05, paths=paths)
    return accuracy.weno_refined_l1(n=128, refine=4, t_end=0.05)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dg3_fq_2048")
    ap.add_argument("--secondary", default="weno_fq_2048,batch64",
                    help="comma-separated workloads measured after the headline into the line's "
                         "'secondary' object ('none' for none)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-refined", action="store_true", help="skip the refined-solution L1 study")
    ap.add_argument("--fp64-only", action="store_true", help="time the FP64 path only")
    ap.add_argument("--batch-policies", default="all,sjf",
                    help="batch workloads: admission policies to run (the first of 'all' or the list is the value)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank, world, local, pg = dist_setup(args.gpus)
    if args.workload.startswith("slab"):
        if rank == 0 and args.impl == "ours":
            print(json.dumps(run_slab(args)), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        if rank == 0:
            out = (run_reference_batch(args) if args.workload.startswith("batch")
                   else run_reference_arm(args, make_workload(args.workload, 0)))
            print(json.dumps(out), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return

    def one(name, primary):
        if name.startswith("batch"):
            return run_batch(name, args, rank, local, world, pg,
                             policies=args.batch_policies if primary else "all",
                             cpu_seconds=8.0 if primary else 4.0)
        return measure_single(name, args, rank, world, local, pg, e2e=not args.no_e2e,
                              cpu_seconds=15.0 if primary else 8.0, refined=not args.no_refined)

    out = one(args.workload, True)
    sec = [n for n in args.secondary.split(",") if n and n not in (args.workload, "none")]
    if sec:
        res = {n: one(n, False) for n in sec}
        if rank == 0:
            out["secondary"] = res
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def parse_batch(name: str) -> tuple[int, int]:
    """batch<N>[_s<steps>]: N problems (default workload: 256), steps each (500)."""
    head, _, tail = name.partition("_s")
    return int(head[len("batch"):] or 256), int(tail or 500)


def batch_cpu_rates(seconds: float = 8.0) -> dict:
    """Reference CPU seconds per cell-step of WENO5 and of DG P=2 (its own
    Persson + Zhang-Shu limiter), each timed on a bounded strip of a 1024^2
    four-quadrant problem with x-slab threads on this host's cores."""
    from oracle.oracle import Reference, reference_available
    from zuikakucfd_b200 import cases
    if not reference_available("faithful"):
        return {}
    cores = max(1, min(os.cpu_count() or 1, 64))
    R = Reference("faithful")
    out = {"cores": cores}
    c = cases.four_quadrant(1024, seed=7)
    lam = c.da / cases.cfl_dt(c, 1.0)
    for key, w in (("weno", dict(case=c, method="weno", order=0, dt=0.4 * c.da / lam)),
                   ("dg2", dict(case=c, method="dg", order=2, dt=0.5 * 0.9 / 10.0 * c.da / lam))):
        st, b, rows = _ref_strip(R, w, cores, 1000.0)
        ms, cells = _ref_slabs(R, w, st, b, 1, cores)
        n = max(1, int(seconds * 1e3 / max(ms, 1.0)))
        ms, cells = _ref_slabs(R, w, st, b, n, cores)
        out[key] = ms * 1e-3 / (cells * n)
        out[key + "_sample"] = f"{n} x updateMesh on a {rows}x1024 strip, {cores} x-slab threads, ISA {R.isa}"
    return out


def run_batch(name: str, args, rank: int, local: int, world: int, pg, policies: str = "all,sjf",
              cpu_seconds: float = 8.0) -> dict | None:
    """Batched serving (one step = one SSP-RK3 step of every running problem):
    N seeded four-quadrant problems, sides uniform in {128, ..., 1024}, half
    WENO5 / half DG P=2, mixed precision, each run `steps` steps at its own CFL
    dt, all through zk_batch (persistent launches, graph-captured steps,
    autotuned tiles).  value = aggregate DOF-updates/s (device time of the run,
    policy "all"); latencies p50/p99 for both admission policies."""
    import torch
    from zuikakucfd_b200.batch import Batch, batch_problems
    nprob, nsteps = parse_batch(name)
    specs = list(batch_problems(nprob, seed=1000 + rank, nsteps=nsteps))
    # pinned host copies of every initial state (the e2e leg uploads from these)
    pinned = [torch.from_numpy(np.ascontiguousarray(s["state"])).pin_memory() for s in specs]
    for s, p in zip(specs, pinned):
        s["state"] = p.numpy()
    in_bytes = sum(p.numel() * 8 for p in pinned)
    cells = sum(int((s["bctype"][3:-3, 3:-3] == 0).sum()) for s in specs)
    # warm-up: the same problems for 3 steps (autotunes every group once; the
    # choice is cached for the process)
    with Batch(policy="all", graph_steps=10, device=local) as b:
        for s in specs:
            b.add(**{**s, "nsteps": 3})
        b.run()
    results = {}
    for policy in policies.split(","):
        barrier(pg)
        with Batch(policy=policy, graph_steps=10, device=local) as b:
            t0 = time.perf_counter()
            ids = [b.add(**s) for s in specs]
            with ClockSampler(local) as clk:
                rep = b.run()
            outs = {}
            for i in ids:  # read every final state back (one buffer per shape)
                shp = b._shapes[i]
                buf = outs.setdefault(shp, torch.empty(shp, dtype=torch.float64).pin_memory())
                from zuikakucfd_b200 import _native as N
                import ctypes as C
                N.check(N.lib().zk_batch_get_state(b._h, i, C.cast(buf.data_ptr(), C.POINTER(C.c_double))))
            wall = time.perf_counter() - t0
            groups = b.groups()
        results[policy] = {"rep": rep, "wall": wall, "clocks": clk.summary(), "groups": groups}
    head = results.get("all") or next(iter(results.values()))
    rep = head["rep"]
    ms = allreduce_max(pg, rep["ms"])
    wall = allreduce_max(pg, head["wall"])
    if rank != 0:
        return None
    peaks = measure_peaks(local)
    flops = 3.0 * sum(int((s["bctype"][3:-3, 3:-3] == 0).sum()) * s["nsteps"] *
                      (1330.0 if s["method"] == "weno" else 5300.0) for s in specs)
    achieved = flops / (ms * 1e-3) / 1e12
    cpu = {"value": None, "skipped": True}
    if not args.no_cpu_baseline and world == 1:
        r = batch_cpu_rates(cpu_seconds)
        if r:
            t_cpu = sum(int((s["bctype"][3:-3, 3:-3] == 0).sum()) * s["nsteps"] *
                        (r["weno"] if s["method"] == "weno" else r["dg2"]) for s in specs)
            cpu = {"value": rep["dof_updates"] / t_cpu, "unit": UNIT, "cores": r["cores"], "kind": "reference",
                   "sample": "per-cell-step cost of the reference's updateMesh measured on bounded strips "
                             f"(WENO5: {r['weno_sample']}; DG P=2: {r['dg2_sample']}), applied to the batch's "
                             "cell-steps", "cell_updates_per_s": rep["cell_updates"] / t_cpu}
    lat = {p: {"p50_ms": v["rep"]["latency_p50_ms"], "p99_ms": v["rep"]["latency_p99_ms"],
               "max_ms": v["rep"]["latency_max_ms"], "device_ms": v["rep"]["ms"],
               "cell_updates_per_s": v["rep"]["cell_updates"] / (v["rep"]["ms"] * 1e-3),
               "done": v["rep"]["done"], "failed": v["rep"]["failed"], "graph_launches": v["rep"]["graph_launches"]}
           for p, v in results.items()}
    out = {"metric": METRIC, "value": world * rep["dof_updates"] / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
           "steps": nsteps, "warmup": 3, "ms_per_step": ms / nsteps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
           "config": {"workload": name, "problems": nprob, "steps_per_problem": nsteps,
                      "desc": f"{nprob} seeded four-quadrant problems, sides uniform in {{128..1024 step 128}}, "
                              "first half WENO5 (CFL 0.4), second half DG P=2 (0.5 x dgSafeDt, reference "
                              "limiter), mixed precision, per-problem dt on the device; policy 'all'",
                      "updated_cells": cells, "l2": "working set %.1f GB >> 126 MB L2" % (in_bytes * 2.5 / 1e9),
                      "parallelism": f"replicas x{world}", "groups": head["groups"]},
           "cell_updates_per_s": world * rep["cell_updates"] / (ms * 1e-3),
           "latency": lat, "clocks": head["clocks"],
           "e2e": {"value": world * rep["dof_updates"] / wall, "unit": UNIT,
                   "h2d_bytes_per_step": in_bytes / nsteps, "d2h_bytes_per_step": in_bytes / nsteps,
                   "what": "zk_batch_add of every problem from pinned host memory + zk_batch_run + "
                           "zk_batch_get_state of every problem, host wall clock, policy 'all'"},
           "gpu_launches": rep["kernel_launches"],
           "roofline": {"bound": "fp32", "achieved": achieved, "peak": peaks["fp32_tflops"], "unit": "TFLOP/s",
                        "frac": achieved / peaks["fp32_tflops"], "traffic": None,
                        "kernel": "whole batch run (all kernels of all groups)",
                        "flops": "3 stages x cell-steps x (1330 WENO5, 5300 DG P=2)",
                        "peak_source": "measured: zk_peak_flops FMA microbenchmark on this GPU"},
           "cpu_baseline": cpu, "peaks": peaks}
    return out


def run_reference_batch(args) -> dict:
    """The reference's CPU updateMesh over the batch's cell-steps, from its
    per-cell-step cost on bounded strips (batch_cpu_rates)."""
    from zuikakucfd_b200.batch import batch_sides
    nprob, nsteps = parse_batch(args.workload)
    r = batch_cpu_rates(4.0)
    if not r:
        return {"impl": "reference", "unavailable": "oracle/_ref (reference built from its sources) missing"}
    sides = batch_sides(nprob, 1000)
    half = nprob // 2
    cells = [(s - 6) ** 2 for s in sides]
    t = sum(c * nsteps * (r["weno"] if i < half else r["dg2"]) for i, c in enumerate(cells))
    dofs = sum(c * nsteps * (4 if i < half else 36) for i, c in enumerate(cells))
    v = dofs / t
    return {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": nsteps, "warmup": 0, "ms_per_step": t * 1e3 / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "problems": nprob},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": "reference",
                             "sample": f"WENO5: {r['weno_sample']}; DG P=2: {r['dg2_sample']}; per-cell-step "
                                       "costs applied to the batch's cell-steps"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_slab(args) -> dict:
    """--workload slab<N>: ms per step of one context over the whole grid
    (zk_step, CUDA events) against N x-slabs of it on this GPU (LocalExchange,
    halos exchanged after every stage), and ms per step of the exchanges alone;
    WENO5 mixed at 2048^2 and DG P=3 mixed at 1024^2, four-quadrant seed 1."""
    import torch
    from zuikakucfd_b200 import cases
    from zuikakucfd_b200.fluid import Solver
    from zuikakucfd_b200.slab import LocalExchange, slab_step, split_arrays
    nslab = int(args.workload[len("slab"):] or 2)
    steps = args.steps

    def one(method, precision, order, n):
        c = cases.four_quadrant(n, seed=1)
        U = c.conserved()
        if method == "dg":
            st = np.zeros((4, (order + 1) ** 2, c.ny, c.nx))
            st[:, 0] = U
            U = st
            dt = 0.5 * 0.9 / (2.0 * (2 * order + 1)) * cases.cfl_dt(c, 1.0)
        else:
            dt = cases.cfl_dt(c, 0.4)

        def make(b, st_):
            s_ = Solver(method=method, order=order, precision=precision)
            s_.set_mesh(c.ny, b.shape[1], c.da, c.gamma, b)
            s_.set_state(st_)
            return s_

        w = make(c.bctype, U)
        w.step(dt, args.warmup)
        ms_whole = w.step_timed(dt, steps) / steps
        w.close()
        solvers = [make(b, s_) for s_, b in split_arrays(U, c.bctype, nslab)]
        try:
            ex = LocalExchange(solvers)
            slab_step(solvers, ex, dt, args.warmup)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(ex.stream)
            slab_step(solvers, ex, dt, steps)
            e1.record(ex.stream)
            e1.synchronize()
            ms_slab = e0.elapsed_time(e1) / steps
            e0.record(ex.stream)
            for _ in range(50):
                for k in (1, 2, 3):
                    ex(k)
            e1.record(ex.stream)
            e1.synchronize()
            ms_ex = e0.elapsed_time(e1) / 50
        finally:
            for s_ in solvers:
                s_.close()
        return {"ms_step_whole": ms_whole, f"ms_step_{nslab}slabs_one_gpu": ms_slab, "ms_exchanges_per_step": ms_ex}

    out = {f"{m}_{p}_P{o}_{n}": one(m, p, o, n) for m, p, o, n in [("weno", "mixed", 2, 2048), ("dg", "mixed", 3, 1024)]}
    return {"workload": args.workload, "slabs": nslab, "steps": steps, "warmup": args.warmup,
            "what": "x-slab decomposition on one GPU vs the whole grid (a diagnostic line, not the metric)",
            "results": out}


def gpu_launches(w, prec) -> int:
    """Kernels of this library launched per step on the headline path."""
    if w["method"] == "weno":
        return 3
    per_stage = 1 if prec == "mixed" else 3
    lim = (w["opts"].get("fp64" if prec == "fp64_fma" else prec, {}) if "fp64" in w["opts"]
           else w["opts"]).get("limiter", "reference")
    return 3 * (per_stage + (1 if lim in ("tvb", "tvb_mlp") else 0))


def open_solver(w, c, U0, precision, device):
    import ctypes as C
    from zuikakucfd_b200 import Solver, _native as N, indicator
    key = "fp64" if precision == "fp64_fma" else precision
    opts = w["opts"].get(key, w["opts"]) if "fp64" in w["opts"] else w["opts"]
    s = Solver(method=w["method"], order=max(w["order"], 1), precision=precision, device=device, **opts)
    s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
    if opts.get("limiter") == "tvb_mlp":
        s.set_indicator()  # the shipped weights and their calibrated screen
    s.set_state(U0)
    return s


if __name__ == "__main__":
    main()
