"""Generate the golden fixtures in tests/golden/ by RUNNING the reference.

The reference ships no tests or golden vectors, so its behaviour is pinned by
executing its own sources: oracle/_ref/libref_*.so are src_WENO/fluid.cpp and
src_DG/fluid.cpp (+ solver.cpp) compiled unmodified against oracle/shim (see
oracle/Makefile).  Two builds are recorded: "strict" (-ffp-contract=off; the
GPU FP64 path must match it bit for bit) and "faithful" (the reference
Makefile's flags, FMA contraction on; matched within a tolerance).

Run where the reference sources are available (this writes only into
tests/golden/):
    make -C oracle ref && python tests/golden/gen_golden.py

Small cases store whole arrays; larger ones store the SHA-256 of the strict
result's bytes (bit-exact check) plus per-field sums and extrema.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle.oracle import REFERENCE_SOURCES, Reference  # noqa: E402
from zuikakucfd_b200 import cases  # noqa: E402

STRICT = Reference("strict")
FAITHFUL = Reference("faithful")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def obstacle_bctype(ny: int, nx: int) -> np.ndarray:
    """Ring of -1 plus an internal -1 block and a lone -1 cell: ghosts whose
    fill sources come from both sweeps, several writers, and unreachable cells."""
    b = np.zeros((ny, nx), np.int32)
    b[:3] = b[-3:] = -1
    b[:, :3] = b[:, -3:] = -1
    b[ny // 2 - 2: ny // 2 + 1, nx // 3: nx // 3 + 4] = -1
    b[5, nx - 7] = -1
    return b


def weno_cases():
    out = {}
    # four quadrants, seeded, odd sizes included
    for (n, ny, seed) in [(24, 24, 3), (23, 37, 11), (7, 7, 5)]:
        c = cases.four_quadrant(n, seed=seed, ny=ny)
        out[f"weno_fq_{n}x{ny}_s{seed}"] = (c.conserved(), c.bctype, c.da, c.gamma, cases.cfl_dt(c, 0.5))
    # internal obstacle ghosts
    c = cases.four_quadrant(26, seed=7)
    out["weno_obstacle_26"] = (c.conserved(), obstacle_bctype(26, 26), c.da, c.gamma, cases.cfl_dt(c, 0.4))
    # frozen-inflow jet (HighMachJet mechanism)
    j = cases.high_mach_jet(40, 20)
    out["weno_jet_40x20"] = (j.conserved(), j.bctype, j.da, j.gamma, 0.3 * j.da / 35.0)
    # no fluid cell at all (every cell a ghost)
    c = cases.four_quadrant(12, seed=2)
    out["weno_allghost_12"] = (c.conserved(), np.full((12, 12), -1, np.int32), c.da, c.gamma, 1e-3)
    return out


def gen_weno(store: dict, meta: dict):
    for name, (U, b, da, g, dt) in weno_cases().items():
        store[f"{name}/U0"] = U
        store[f"{name}/bct"] = b
        meta[name] = {"da": da, "gamma": g, "dt": dt, "steps": [1, 10]}
        for n in (1, 10):
            store[f"{name}/strict_{n}"] = STRICT.weno_step(U, b, da, g, dt, n)
            store[f"{name}/faithful_{n}"] = FAITHFUL.weno_step(U, b, da, g, dt, n)
        Uf, dU = STRICT.weno_rhs(U, b, da, g, dt)
        store[f"{name}/rhs_U"] = Uf
        store[f"{name}/rhs_dU"] = dU
        meta[name]["max_speed"] = STRICT.weno_max_speed(U, b, da, g)
        meta[name]["max_speed_10"] = STRICT.weno_max_speed(store[f"{name}/strict_10"], b, da, g)
        store[f"{name}/prim_10"] = STRICT.weno_recover(store[f"{name}/strict_10"], b, da, g)

    # periodic smooth wave through the harness's periodic RK loop
    w = cases.smooth_wave(16)
    U = w.conserved()
    dt = 0.4 * w.da / 2.5
    store["weno_wave_16/U0"] = U
    store["weno_wave_16/bct"] = w.bctype
    meta["weno_wave_16"] = {"da": w.da, "gamma": w.gamma, "dt": dt, "steps": [5], "periodic": True}
    store["weno_wave_16/strict_5"] = STRICT.weno_step(U, w.bctype, w.da, w.gamma, dt, 5, periodic=True)
    store["weno_wave_16/faithful_5"] = FAITHFUL.weno_step(U, w.bctype, w.da, w.gamma, dt, 5, periodic=True)


def gen_weno_large(meta: dict, store: dict):
    """The reference's own 2D-Riemann case (256x256) and a 128^2 seeded case:
    hashes of the strict results (bit-exact) plus a few sampled rows."""
    ref_case = REFERENCE_SOURCES / "2D-Riemann"
    U, b, da, g = STRICT.weno_load_case(ref_case)
    dt = 0.5 * da / STRICT.weno_max_speed(U, b, da, g)
    store["riemann256/U0"] = U   # the reference's own input case (piecewise constant: compresses to KBs)
    store["riemann256/bct"] = b
    entry = {"da": da, "gamma": g, "dt": dt, "steps": 20}
    S = STRICT.weno_step(U, b, da, g, dt, 20)
    F = FAITHFUL.weno_step(U, b, da, g, dt, 20)
    entry["strict_sha256"] = sha(S)
    entry["strict_sums"] = S.sum(axis=(1, 2)).tolist()
    entry["faithful_vs_strict_rel_linf"] = float((np.abs(F - S).max(axis=(1, 2)) / np.abs(S).max(axis=(1, 2))).max())
    store["riemann256/strict_20_rows"] = S[:, ::17].copy()
    store["riemann256/faithful_20_rows"] = F[:, ::17].copy()
    entry["max_speed"] = STRICT.weno_max_speed(U, b, da, g)
    meta["riemann256"] = entry

    c = cases.four_quadrant(128, seed=42)
    U = c.conserved()
    dt = cases.cfl_dt(c, 0.5)
    S = STRICT.weno_step(U, c.bctype, c.da, c.gamma, dt, 50)
    F = FAITHFUL.weno_step(U, c.bctype, c.da, c.gamma, dt, 50)
    meta["weno_fq128_s42"] = {"n": 128, "seed": 42, "dt": dt, "steps": 50, "strict_sha256": sha(S),
                              "strict_sums": S.sum(axis=(1, 2)).tolist(),
                              "faithful_vs_strict_rel_linf":
                                  float((np.abs(F - S).max(axis=(1, 2)) / np.abs(S).max(axis=(1, 2))).max())}
    store["weno_fq128_s42/strict_50_rows"] = S[:, ::13].copy()


def dg_cases(P: int):
    out = {}
    c = cases.four_quadrant(20, seed=5)
    out["fq20"] = (c.dg_state(P), c.bctype, c.da, c.gamma)
    c2 = cases.four_quadrant(17, seed=9, ny=23)
    out["fq17x23"] = (c2.dg_state(P), c2.bctype, c2.da, c2.gamma)
    # slip walls on the top/bottom ring, copy ghosts left/right, internal slip block
    c3 = cases.four_quadrant(22, seed=13)
    b = c3.bctype.copy()
    b[:3, 3:-3] = 1
    b[-3:, 3:-3] = 1
    b[9:12, 9:12] = 1
    out["slip22"] = (c3.dg_state(P), b, c3.da, c3.gamma)
    # near-vacuum strip: drives the Zhang-Shu density / pressure limits
    c4 = cases.four_quadrant(18, seed=21)
    d = c4.dg_state(P)
    rng = np.random.default_rng(100 + P)
    d[:, 1:] = rng.normal(0.0, 0.3, d[:, 1:].shape)
    d[0, 0, 6:9] = 2e-5
    d[3, 0, 6:9] = 1e-5
    out["vacuum18"] = (d, c4.bctype, c4.da, c4.gamma)
    return out


def gen_dg(store: dict, meta: dict):
    for P in (1, 2, 3):
        for cname, (d, b, da, g) in dg_cases(P).items():
            name = f"dg{P}_{cname}"
            lam = STRICT.dg_max_speed(P, d, b, da, g)
            dt = 0.5 * STRICT.dg_safe_dt(P, lam, da)
            store[f"{name}/dof0"] = d
            store[f"{name}/bct"] = b
            meta[name] = {"P": P, "da": da, "gamma": g, "dt": dt, "max_speed": lam}
            store[f"{name}/strict_3"] = STRICT.dg_step(P, d, b, da, g, dt, 3)
            store[f"{name}/faithful_3"] = FAITHFUL.dg_step(P, d, b, da, g, dt, 3)
            x, dU = STRICT.dg_rhs(P, d, b, da, g)
            store[f"{name}/rhs_dof"] = x
            store[f"{name}/rhs_dU"] = dU
            store[f"{name}/limit"] = STRICT.dg_limit(P, d, b, da, g)
            meta[name]["max_speed_3"] = STRICT.dg_max_speed(P, store[f"{name}/strict_3"], b, da, g)
        # periodic smooth wave
        w = cases.smooth_wave(12)
        d = w.dg_state(P)
        dt = 0.5 * STRICT.dg_safe_dt(P, 2.6, w.da)
        name = f"dg{P}_wave12"
        store[f"{name}/dof0"] = d
        store[f"{name}/bct"] = w.bctype
        meta[name] = {"P": P, "da": w.da, "gamma": w.gamma, "dt": dt, "periodic": True}
        store[f"{name}/strict_3"] = STRICT.dg_step(P, d, w.bctype, w.da, w.gamma, dt, 3, periodic=True)
        store[f"{name}/faithful_3"] = FAITHFUL.dg_step(P, d, w.bctype, w.da, w.gamma, dt, 3, periodic=True)


def gen_points(store: dict, meta: dict):
    """Riemann-solver point vectors: random states plus vacuum / negative
    pressure / NaN-guard edge cases."""
    rng = np.random.default_rng(2024)
    n = 400
    rho = np.concatenate([rng.uniform(0.05, 3, (n, 2)), np.array([[1e-14, 1.0], [1.0, 1e-14], [0.0, 0.0],
                                                              [2e-6, 3e-6], [1.0, 1.0]])])
    m = rho.shape[0]
    vel = rng.uniform(-3, 3, (m, 2, 2))
    p = np.concatenate([rng.uniform(0.01, 3, (n, 2)), np.array([[1.0, 1.0], [1.0, 1.0], [0.0, 0.0],
                                                            [1e-7, 1e-7], [-1.0, 2.0]])])
    g = 1.4
    L = np.stack([rho[:, 0], rho[:, 0] * vel[:, 0, 0], rho[:, 0] * vel[:, 0, 1],
                  p[:, 0] / (g - 1) + 0.5 * rho[:, 0] * (vel[:, 0] ** 2).sum(1)], 1)
    R = np.stack([rho[:, 1], rho[:, 1] * vel[:, 1, 0], rho[:, 1] * vel[:, 1, 1],
                  p[:, 1] / (g - 1) + 0.5 * rho[:, 1] * (vel[:, 1] ** 2).sum(1)], 1)
    store["points/L"] = L
    store["points/R"] = R
    store["points/hllc_weno"] = np.array([STRICT.hllc_weno(L[k], R[k], g) for k in range(m)])
    store["points/hllc_dg"] = np.array([STRICT.hllc_dg(L[k], R[k], g) for k in range(m)])
    store["points/hlle_dg"] = np.array([STRICT.hlle_dg(L[k], R[k], g) for k in range(m)])
    meta["points"] = {"gamma": g}
    # basis values phi2(m, xi, eta) at P = 1..3
    pts = np.array([-1.0, -0.7745966692414834, -0.3, 0.0, 0.5773502691896257, 1.0])
    for P in (1, 2, 3):
        nm = (P + 1) ** 2
        store[f"points/phi2_P{P}"] = np.array([[[STRICT.phi2(P, mm, a, b) for b in pts] for a in pts]
                                               for mm in range(nm)])
    store["points/phi2_pts"] = pts


def gen_muscl(store: dict, meta: dict):
    """The reference's muscl_reconstruct (src_WENO/fluid.cpp:203-225) on
    seeded stencils (UL2, UL1, UR1, UR2) with sign changes, equal neighbours,
    zeros and opposite slopes, for limiters 0 (minmod), 1 (van Leer), 2
    (superbee), strict and Makefile-faithful builds."""
    rng = np.random.default_rng(2025)
    st = rng.normal(0.0, 1.0, (600, 4))
    st[::7, 1] = st[::7, 0]
    st[::11, 2] = st[::11, 1]
    st[::13] = 0.0
    st[::17, 3] = -st[::17, 2]
    st[::19] = np.array([1.0, 2.0, 4.0, 8.0])
    store["muscl/stencils"] = st
    for lim in (0, 1, 2):
        store[f"muscl/strict_L{lim}"] = STRICT.muscl(st, lim)
        store[f"muscl/faithful_L{lim}"] = FAITHFUL.muscl(st, lim)
    meta["muscl"] = {"limiters": {"0": "minmod", "1": "van Leer", "2": "superbee"}}


def main():
    store: dict[str, np.ndarray] = {}
    meta: dict = {}
    gen_weno(store, meta)
    gen_weno_large(meta, store)
    gen_dg(store, meta)
    gen_points(store, meta)
    gen_muscl(store, meta)
    np.savez_compressed(HERE / "reference_golden.npz", **store)
    (HERE / "reference_golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    sz = (HERE / "reference_golden.npz").stat().st_size
    print(f"wrote {len(store)} arrays, {sz / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
