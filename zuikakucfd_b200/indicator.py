"""The learned troubled-cell indicator of the DG TVB limiter.

A 40 -> 32 -> 32 -> 32 -> 1 GELU MLP (the layout is documented in
include/zuikaku.h) trained on labels the plain TVB-minmod indicator produces
on seeded four-quadrant runs, then used by DG contexts with
limiter="tvb_mlp": only the cells it flags take the characteristic-limiting
branch.  Its inputs for an RK stage's output are the output's rho and E modes
and the means of the stage's input, which the mixed-precision stage kernel
holds in its tile, so the indicator runs inside that kernel.  Training runs
on the GPU through the library's own forward/backward/Adam kernels
(zk_mlp_train); nothing here runs on the CPU but data plumbing.

    python -m zuikakucfd_b200.indicator train --out weights.npz
    python -m zuikakucfd_b200.indicator eval --weights weights.npz

The trained weights shipped with the package live in
zuikakucfd_b200/data/indicator_p3.npz (see DEFAULT_WEIGHTS).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import _native as N
from . import cases

DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "indicator_p3.npz"
NPARAM, NIN = N.MLP_NPARAM, N.MLP_IN


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial weights, zero biases (flat FP32 block)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, np.sqrt(2.0 / 40), (32, 40)), np.zeros(32), rng.normal(0, np.sqrt(2.0 / 32), (32, 32)),
             np.zeros(32), rng.normal(0, np.sqrt(2.0 / 32), (32, 32)), np.zeros(32),
             rng.normal(0, np.sqrt(1.0 / 32), 32), np.zeros(1)]
    return np.concatenate([np.ravel(a) for a in parts]).astype(np.float32)


def features_and_labels(solver) -> tuple[np.ndarray, np.ndarray]:
    """(features[ny*nx][40], TVB labels[ny*nx]) of a DG Solver's current state."""
    n = solver.ny * solver.nx
    X = np.zeros((n, NIN), np.float32)
    y = np.zeros(n, np.uint8)
    N.check(N.lib().zk_indicator_features(solver._h, _fp(X), y.ctypes.data_as(C.POINTER(C.c_uint8))))
    return X, y


def stage_features_and_labels(solver, stage: int) -> tuple[np.ndarray, np.ndarray]:
    """(features[ny*nx][40], TVB labels[ny*nx]) of the output of RK stage
    `stage`, which solver.stage(dt, stage) has just computed: the output's
    modes with the stage input's means, labelled by the plain TVB indicator
    on the output."""
    n = solver.ny * solver.nx
    X = np.zeros((n, NIN), np.float32)
    y = np.zeros(n, np.uint8)
    N.check(N.lib().zk_indicator_stage_features(solver._h, int(stage), _fp(X), y.ctypes.data_as(C.POINTER(C.c_uint8))))
    return X, y


def generate_dataset(n_runs: int = 64, n: int = 512, order: int = 3, steps: int = 160, snapshots: int = 4,
                     per_run: int = 160_000, seed0: int = 5000, M: float = 50.0, device: int = 0,
                     cfl_frac: float = 0.5, verbose: bool = True):
    """Seeded four-quadrant runs advanced with the plain TVB limiter; at
    `snapshots` times the state is advanced one unlimited FP64 step, stage by
    stage, and every updated cell of each stage's output is a sample: its
    features (the output's modes, the stage input's means) labelled by the
    TVB indicator on the output.  Per run all troubled cells are kept and the
    rest is filled with randomly chosen smooth cells up to `per_run` samples.
    Runs whose state goes non-finite are dropped.  Returns X[N][40], y[N],
    metadata."""
    from .fluid import Solver
    rng = np.random.default_rng(seed0)
    Xs, ys, used = [], [], []
    t0 = time.time()
    for r in range(n_runs):
        seed = seed0 + r
        c = cases.four_quadrant(n, seed=seed)
        lam = c.da / cases.cfl_dt(c, 1.0)
        dt = cfl_frac * 0.9 / (2.0 * (2 * order + 1)) * c.da / lam
        upd = np.zeros((c.ny, c.nx), bool)
        upd[3:-3, 3:-3] = c.bctype[3:-3, 3:-3] == 0
        upd = upd.ravel()
        with Solver(method="dg", order=order, precision="mixed", limiter="tvb", tvb_M=M, device=device) as s, \
                Solver(method="dg", order=order, precision="fp64", limiter="none", tvb_M=M, device=device) as raw:
            s.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
            raw.set_mesh(c.ny, c.nx, c.da, c.gamma, c.bctype)
            s.set_state(c.dg_state(order))
            rx, ry = [], []
            ok = True
            every = max(1, steps // snapshots)
            for k in range(snapshots):
                s.step(dt, every)
                st = s.get_state()
                if s.status_word() or not np.isfinite(st).all():
                    ok = False
                    break
                raw.set_state(st)
                for stage in (1, 2, 3):
                    raw.stage(dt, stage)
                    X, y = stage_features_and_labels(raw, stage)
                    rx.append(X[upd])
                    ry.append(y[upd])
            if not ok or not rx:
                continue
            X = np.concatenate(rx)
            y = np.concatenate(ry)
            pos = np.flatnonzero(y)
            neg = np.flatnonzero(y == 0)
            keep_neg = rng.choice(neg, size=min(len(neg), max(0, per_run - len(pos))), replace=False)
            sel = np.concatenate([pos, keep_neg])
            Xs.append(X[sel])
            ys.append(y[sel])
            used.append(seed)
        if verbose and (r % 8 == 7 or r == n_runs - 1):
            print(f"  runs {r + 1}/{n_runs}: {sum(len(a) for a in ys)} samples, {time.time() - t0:.1f}s", flush=True)
    X = np.concatenate(Xs)
    y = np.concatenate(ys)
    meta = {"runs": len(used), "seeds": used, "grid": n, "order": order, "steps": steps, "snapshots": snapshots,
            "M": M, "samples": int(len(y)), "positives": int(y.sum()), "features": "stage output modes, stage input means",
            "seconds": time.time() - t0}
    return X, y, meta


def train(X: np.ndarray, y: np.ndarray, epochs: int = 6, batch: int = 4096, lr: float = 2e-3,
          pos_weight: float | None = None, seed: int = 0, device: int = 0, params: np.ndarray | None = None):
    """Train on the GPU (zk_mlp_train); returns (params, per-epoch mean loss)."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.uint8)
    if pos_weight is None:
        pos = max(1, int(y.sum()))
        pos_weight = float(min(20.0, (len(y) - pos) / pos))
    p = np.array(init_params(seed) if params is None else params, np.float32)
    losses = np.zeros(epochs, np.float32)
    N.check(N.lib().zk_mlp_train(device, _fp(X), y.ctypes.data_as(C.POINTER(C.c_uint8)), len(y), _fp(p), epochs,
                                 batch, lr, pos_weight, seed, _fp(losses)))
    return p, losses


def logits(params: np.ndarray, X: np.ndarray, bf16: bool = True, device: int = 0) -> np.ndarray:
    X = np.ascontiguousarray(X, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    out = np.zeros(len(X), np.float32)
    N.check(N.lib().zk_mlp_forward(device, _fp(X), len(X), _fp(p), int(bf16), _fp(out)))
    return out


def deviation(X: np.ndarray) -> np.ndarray:
    """Largest |feature| of each row, its deviation from a constant state's
    (all features 0): the screen's quantity."""
    return np.abs(X).max(axis=1)


def calibrate_screen(X: np.ndarray, y: np.ndarray, margin: float = 0.5) -> dict:
    """The screen: `margin` x the smallest deviation of any TVB-troubled
    training cell, so that no troubled training cell is screened out."""
    d = deviation(X)
    pos = y.astype(bool)
    tau = float(margin * d[pos].min()) if pos.any() else -1.0
    return {"screen": tau, "pos_dev_min": float(d[pos].min()) if pos.any() else None,
            "pos_dev_q1e-4": float(np.quantile(d[pos], 1e-4)) if pos.any() else None,
            "neg_screened": float((d[~pos] <= tau).mean()) if (~pos).any() else None}


def agreement(params: np.ndarray, X: np.ndarray, y: np.ndarray, bf16: bool = True, device: int = 0,
              screen: float = -1.0) -> dict:
    """Flag agreement with the TVB labels: accuracy, missed-discontinuity rate
    (TVB-troubled cells the indicator does not flag), false-flag rate.  With a
    screen (>= 0) the indicator flags a cell when its deviation exceeds the
    screen and the network's logit is positive."""
    f = logits(params, X, bf16, device) > 0
    if screen >= 0:
        f &= deviation(X) > screen
    t = y.astype(bool)
    tp = int((f & t).sum())
    return {"accuracy": float((f == t).mean()), "missed_rate": float(((~f) & t).sum() / max(1, t.sum())),
            "false_flag_rate": float((f & ~t).sum() / max(1, (~t).sum())),
            "precision": float(tp / max(1, f.sum())), "flag_rate": float(f.mean()), "n": int(len(y))}


def load_screen(path=None) -> float:
    """The screen calibrated with the weights (-1 when they carry none)."""
    z = np.load(path or DEFAULT_WEIGHTS)
    meta = json.loads(str(z["meta"])) if "meta" in z.files else {}
    return float(meta.get("screen", -1.0))


def save(path, params, meta: dict | None = None) -> None:
    np.savez(path, params=np.asarray(params, np.float32), meta=json.dumps(meta or {}))


def load(path=None) -> np.ndarray:
    z = np.load(path or DEFAULT_WEIGHTS)
    p = np.asarray(z["params"], np.float32)
    if p.size != NPARAM:
        raise ValueError(f"{path}: expected {NPARAM} parameters, found {p.size}")
    return p


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="train / evaluate the learned troubled-cell indicator")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    t.add_argument("--recalibrate", default=None,
                   help="keep the weights of this file and only calibrate the screen on fresh data")
    t.add_argument("--runs", type=int, default=64)
    t.add_argument("--grid", type=int, default=512)
    t.add_argument("--per-run", type=int, default=160_000)
    t.add_argument("--epochs", type=int, default=6)
    t.add_argument("--holdout-runs", type=int, default=4)
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=None)
    e.add_argument("--runs", type=int, default=4)
    e.add_argument("--grid", type=int, default=512)
    a = ap.parse_args(argv)
    if a.cmd == "train" and a.recalibrate:
        p = load(a.recalibrate)
        old = json.loads(str(np.load(a.recalibrate)["meta"]))
        X, y, _ = generate_dataset(n_runs=a.runs, n=a.grid, per_run=a.per_run)
        old.update(calibrate_screen(X, y))
        Xh, yh, _ = generate_dataset(n_runs=a.holdout_runs, n=a.grid, per_run=a.per_run, seed0=9000)
        old["holdout_with_screen"] = agreement(p, Xh, yh, screen=old["screen"])
        old["holdout_screened"] = float((deviation(Xh) <= old["screen"]).mean())
        save(a.out, p, old)
        print(json.dumps({k: old[k] for k in ("screen", "pos_dev_min", "pos_dev_q1e-4", "neg_screened",
                                               "holdout_with_screen", "holdout_screened")}), flush=True)
        return 0
    if a.cmd == "train":
        X, y, meta = generate_dataset(n_runs=a.runs, n=a.grid, per_run=a.per_run)
        print(json.dumps({k: v for k, v in meta.items() if k != "seeds"}), flush=True)
        t0 = time.time()
        p, losses = train(X, y, epochs=a.epochs)
        meta["train_seconds"] = time.time() - t0
        meta.update(calibrate_screen(X, y))
        Xh, yh, mh = generate_dataset(n_runs=a.holdout_runs, n=a.grid, per_run=a.per_run, seed0=9000)
        ag = agreement(p, Xh, yh)
        ags = agreement(p, Xh, yh, screen=meta["screen"])
        meta.update({"epoch_loss": losses.tolist(), "holdout": ag, "holdout_with_screen": ags,
                     "holdout_screened": float((deviation(Xh) <= meta["screen"]).mean()),
                     "holdout_seeds": mh["seeds"]})
        save(a.out, p, meta)
        print(json.dumps({k: meta[k] for k in ("epoch_loss", "holdout", "holdout_with_screen", "screen",
                                                "pos_dev_min", "pos_dev_q1e-4", "neg_screened",
                                                "holdout_screened")}), flush=True)
    else:
        p = load(a.weights)
        Xh, yh, _ = generate_dataset(n_runs=a.runs, n=a.grid, seed0=9000)
        print(json.dumps(agreement(p, Xh, yh)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
