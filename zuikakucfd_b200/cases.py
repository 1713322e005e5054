"""Seeded initial conditions in the reference's case format.

Conventions follow the reference's generator notebook (gen.ipynb, cells 0-1):
``da = L / nx``; row 0 is the TOP of the domain (``yc = y_max - (i + 0.5) da``)
and column 0 the left (``xc = x_min + (j + 0.5) da``); the boundary ring lies
inside the ``ny x nx`` grid; files are ``params.txt`` ("nx ny da gamma") plus
row-major text matrices ``rho/u/v/p/bctype.dat``.

Randomised states use ``numpy.random.default_rng(seed)``, drawing the four
quadrants in the fixed order NE, NW, SW, SE and (rho, u, v, p) within each.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np


@dataclass
class Case:
    name: str
    ny: int
    nx: int
    da: float
    gamma: float
    rho: np.ndarray
    u: np.ndarray
    v: np.ndarray
    p: np.ndarray
    bctype: np.ndarray
    periodic: bool = False
    seed: int | None = None

    def conserved(self) -> np.ndarray:
        """U[4][ny][nx] = rho, rho u, rho v, E (src_WENO/fluid.cpp:86-93)."""
        r, u, v, p, g = self.rho, self.u, self.v, self.p, self.gamma
        return np.stack([r, r * u, r * v, p / (g - 1.0) + 0.5 * r * (u * u + v * v)])

    def dg_state(self, order: int) -> np.ndarray:
        """dof[4][NM][ny][nx] with mode 0 = the cell values (initDGModes,
        src_DG/fluid.cpp:173-182)."""
        nm = (order + 1) ** 2
        d = np.zeros((4, nm, self.ny, self.nx))
        d[:, 0] = self.conserved()
        return d

    @property
    def fluid_cells(self) -> int:
        """Cells the RHS updates: bctype 0 inside [3, ny-3) x [3, nx-3)."""
        return int((self.bctype[3:-3, 3:-3] == 0).sum())


def _ring(ny: int, nx: int, width: int = 3, code: int = -1) -> np.ndarray:
    b = np.zeros((ny, nx), np.int32)
    b[:width, :] = code
    b[-width:, :] = code
    b[:, :width] = code
    b[:, -width:] = code
    return b


def four_quadrant(n: int = 256, seed: int = 0, gamma: float = 1.4, ny: int | None = None,
                  split: float = 0.5, ring_code: int = -1, ring_outside: bool = False) -> Case:
    """Four constant quadrants split at (split, split) by cell centre; each
    quadrant rho,p ~ U[0.1,2], u,v ~ U[-1,1]; 3-cell ring.

    Default (the notebook's convention): the n x ny grid, ring included, spans
    [0,1] x [0, ny/n] with da = 1/n.  ring_outside=True: the n x ny cells are
    the INTERIOR on [0,1] x [0, ny/n] (da = 1/n) and the ring lies outside it,
    so grids of different resolution cover the same physical interior."""
    nx = int(n)
    ny = int(ny or n)
    da = 1.0 / nx
    rng = np.random.default_rng(seed)
    # NE, NW, SW, SE; (rho, u, v, p) each
    q = []
    for _ in range(4):
        rho = rng.uniform(0.1, 2.0)
        u = rng.uniform(-1.0, 1.0)
        v = rng.uniform(-1.0, 1.0)
        p = rng.uniform(0.1, 2.0)
        q.append((rho, u, v, p))
    if ring_outside:
        gx, gy = nx + 6, ny + 6
        xc = (np.arange(gx) - 3 + 0.5) * da
        yc = ny * da - (np.arange(gy) - 3 + 0.5) * da
    else:
        gx, gy = nx, ny
        xc = (np.arange(nx) + 0.5) * da
        yc = ny * da - (np.arange(ny) + 0.5) * da
    X, Y = np.meshgrid(xc, yc)
    east, north = X >= split, Y >= split
    idx = np.where(north & east, 0, np.where(north, 1, np.where(east, 3, 2)))
    tab = np.array(q)
    f = tab[idx]
    return Case(f"four_quadrant_{gx}x{gy}_s{seed}", gy, gx, da, gamma, f[..., 0], f[..., 1],
                f[..., 2], f[..., 3], _ring(gy, gx, 3, ring_code), seed=seed)


def riemann_config(n: int = 512, gamma: float = 1.4, ny: int | None = None, split: float = 0.85) -> Case:
    """The generator notebook's fixed four-quadrant Riemann configuration
    (gen.ipynb cell 0): interfaces at x = y = split on [0,1]^2 (row 0 on top),
    NE (1.5, 0, 0, 1.5), NW (0.5323, 1.206, 0, 0.3), SW (0.138, 1.206, -1.206,
    0.029), SE (0.5323, 0, -1.206, 0.3) as (rho, u, v, p); 3-cell -1 ring.
    The reference's shipped 2D-Riemann case is this configuration at n = 256
    with split = 0.8 (its interfaces lie between columns 204/205 and rows
    50/51); the notebook's default is 0.85."""
    nx = int(n)
    ny = int(ny or n)
    da = 1.0 / nx
    xc = (np.arange(nx) + 0.5) * da
    yc = 1.0 - (np.arange(ny) + 0.5) * da
    X, Y = np.meshgrid(xc, yc)
    east, north = X >= split, Y >= split
    tab = np.array([(1.5, 0.0, 0.0, 1.5), (0.5323, 1.206, 0.0, 0.3), (0.138, 1.206, -1.206, 0.029),
                    (0.5323, 0.0, -1.206, 0.3)])
    f = tab[np.where(north & east, 0, np.where(north, 1, np.where(east, 3, 2)))]
    return Case(f"riemann_config_{nx}x{ny}", ny, nx, da, gamma, f[..., 0], f[..., 1], f[..., 2], f[..., 3],
                _ring(ny, nx, 3, -1))


def center_detonation(n: int = 1024, gamma: float = 1.4, domain: float = 2000.0, R0: float = 10.0,
                      rho_in: float = 0.1, p_in: float = 1e10, rho_out: float = 1.225,
                      p_out: float = 101325.0) -> Case:
    """The generator notebook's centre detonation (gen.ipynb cell 1), SI units:
    a disc of radius R0 at the centre of [0, domain]^2 holding (rho_in, p_in)
    in air at rest (rho_out, p_out); 2-cell -1 ring, as the notebook writes."""
    nx = ny = int(n)
    da = domain / nx
    xc = (np.arange(nx) + 0.5) * da
    yc = domain - (np.arange(ny) + 0.5) * da
    X, Y = np.meshgrid(xc, yc)
    inside = (X - domain / 2.0) ** 2 + (Y - domain / 2.0) ** 2 <= R0 * R0
    rho = np.where(inside, rho_in, rho_out)
    p = np.where(inside, p_in, p_out)
    zero = np.zeros((ny, nx))
    return Case(f"center_detonation_{nx}", ny, nx, da, gamma, rho, zero.copy(), zero.copy(), p,
                _ring(ny, nx, 2, -1))


def smooth_wave(n_interior: int = 1024, gamma: float = 1.4, amplitude: float = 0.2,
                length: float = 2.0, u: float = 1.0, v: float = 1.0) -> Case:
    """rho = 1 + a sin(pi (x + y)), u = v = 1, p = 1 on [0, length]^2, periodic:
    n_interior^2 fluid cells plus a 3-cell ring marked -3 holding the periodic
    images.  Exact solution at time t: smooth_wave_exact (steady for u = v = 1
    in the solvers' orientation; periodic in t with period `length` either
    way)."""
    n = int(n_interior)
    h = length / n
    N = n + 6
    k = np.arange(N)
    xc = ((k - 3) % n + 0.5) * h             # periodic image coordinate
    yc = length - ((k - 3) % n + 0.5) * h
    X, Y = np.meshgrid(xc, yc)
    rho = 1.0 + amplitude * np.sin(np.pi * (X + Y))
    one = np.ones((N, N))
    return Case(f"smooth_wave_{n}", N, N, h, gamma, rho, u * one, v * one, one.copy(),
                _ring(N, N, 3, -3), periodic=True)


def smooth_wave_exact(case: Case, t: float, amplitude: float = 0.2, length: float = 2.0) -> np.ndarray:
    """Cell-centre density of the translated wave at time t (interior cells).

    Both reference solvers difference the y fluxes along increasing row index
    (the face below minus the face above, src_WENO/fluid.cpp:454-460; the DG
    bottom face is eta = +1 towards row i+1), so v is the velocity towards
    increasing row, i.e. downwards in a case file whose row 0 is the top: the
    exact solution is rho0(x - u t, y + v t).  With u = v = 1 the wave
    1 + a sin(pi (x + y)) moves along its own crests and is steady; v = -1
    translates it along the diagonal."""
    n = case.nx - 6
    h = length / n
    c = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(c, length - c)
    u, v = float(case.u.flat[0]), float(case.v.flat[0])
    return 1.0 + amplitude * np.sin(np.pi * ((X - u * t) + (Y + v * t)))


def high_mach_jet(nx: int = 2048, ny: int = 1024, gamma: float = 5.0 / 3.0, u_jet: float = 30.0,
                  rho_jet: float = 5.0, rho_amb: float = 0.5, p_amb: float = 0.4127,
                  half_width: float = 0.05) -> Case:
    """Jet on [0,1] x [-0.25,0.25] (da = 1/nx).  Following the HighMachJet
    case: columns 0-2 of the rows inside the ring are bctype-0 cells that the
    RHS loop never updates (frozen inflow); the band |yc| < half_width carries
    (rho_jet, u_jet); -1 ring elsewhere."""
    da = 1.0 / nx
    y_top = ny * da / 2.0
    yc = y_top - (np.arange(ny) + 0.5) * da
    rho = np.full((ny, nx), rho_amb)
    u = np.zeros((ny, nx))
    v = np.zeros((ny, nx))
    p = np.full((ny, nx), p_amb)
    band = np.abs(yc) < half_width
    rho[band, :3] = rho_jet
    u[band, :3] = u_jet
    b = _ring(ny, nx, 3, -1)
    b[3:-3, :3] = 0
    return Case(f"high_mach_jet_{nx}x{ny}", ny, nx, da, gamma, rho, u, v, p, b)


def write_case(case: Case, folder: str | os.PathLike, fmt: str = "%.17e") -> Path:
    """Write params.txt + rho/u/v/p/bctype.dat in the reference's format."""
    d = Path(folder)
    d.mkdir(parents=True, exist_ok=True)
    (d / "params.txt").write_text(f"{case.nx} {case.ny} {case.da:.17e} {case.gamma!r}\n")
    for name in ("rho", "u", "v", "p"):
        np.savetxt(d / f"{name}.dat", getattr(case, name), fmt=fmt, delimiter=" ")
    np.savetxt(d / "bctype.dat", case.bctype, fmt="%d", delimiter=" ")
    return d


def cfl_dt(case: Case, cfl: float = 0.5) -> float:
    """dt = cfl * da / lambda0, lambda0 = max over ALL cells of |u| + a (the
    reference's computeMaxSpeed rule, src_WENO/fluid.cpp:539-553)."""
    a = np.sqrt(case.gamma * case.p / case.rho)
    lam = float(np.max(np.sqrt(case.u ** 2 + case.v ** 2) + a))
    return cfl * case.da / lam


def smooth_wave_modes(case: Case, order: int, t: float = 0.0, amplitude: float = 0.2,
                      length: float = 2.0, nq: int = 6) -> np.ndarray:
    """L2 projection of the translated smooth wave at time t onto the DG
    basis, dof[4][NM][ny][nx] (ghost ring included: periodic images).

    The reference initialises mode 0 with the cell-centre value only
    (src_DG/fluid.cpp:173-182), an O(h^2) start that hides the scheme's order;
    this projection is the accuracy-study initial condition.  Reference-cell
    coordinates follow the reference's face convention: xi = +1 is the right
    face, eta = +1 the face towards row i+1 (downwards, decreasing y).
    Modes: d_m = (2px+1)(2py+1)/4 * integral of u(xi, eta) P_px(xi) P_py(eta),
    m = px (P+1) + py, by an nq x nq Gauss rule."""
    from numpy.polynomial.legendre import leggauss, legval
    P = int(order)
    NQ = P + 1
    nm = NQ * NQ
    g = case.gamma
    x, w = leggauss(nq)
    n = case.nx - 6
    h = length / n
    k = np.arange(case.nx)
    xc = ((k - 3) % n + 0.5) * h
    yc = length - ((np.arange(case.ny) - 3) % n + 0.5) * h
    Pv = np.array([legval(x, np.eye(NQ)[p]) for p in range(NQ)])  # [p][q]
    # density at the nq x nq points of every cell: rho[i, j, a, b]
    X = xc[None, :, None, None] + 0.5 * h * x[None, None, :, None]
    Y = yc[:, None, None, None] - 0.5 * h * x[None, None, None, :]
    u, v = float(case.u.flat[0]), float(case.v.flat[0])
    rho = 1.0 + amplitude * np.sin(np.pi * ((X - u * t) + (Y + v * t)))  # y + v t: see smooth_wave_exact
    rm = np.zeros((nm,) + rho.shape[:2])
    for px in range(NQ):
        for py in range(NQ):
            wt = (w * Pv[px])[:, None] * (w * Pv[py])[None, :]
            rm[px * NQ + py] = (2 * px + 1) * (2 * py + 1) / 4.0 * np.einsum("ijab,ab->ij", rho, wt)
    d = np.zeros((4, nm, case.ny, case.nx))
    d[0] = rm
    d[1] = u * rm                      # rho u (u, v, p constant)
    d[2] = v * rm                      # rho v
    d[3] = 0.5 * (u * u + v * v) * rm  # E = p/(gamma-1) + rho (u^2+v^2)/2
    d[3, 0] += float(case.p.flat[0]) / (g - 1.0)
    return d


GENERATORS = {
    "four_quadrant": lambda a: four_quadrant(a.n, seed=a.seed),
    "riemann_config": lambda a: riemann_config(a.n),
    "center_detonation": lambda a: center_detonation(a.n),
    "smooth_wave": lambda a: smooth_wave(a.n),
    "high_mach_jet": lambda a: high_mach_jet(a.n, a.n // 2),
}


def main(argv=None) -> int:
    """Write a case folder in the reference's format:
    python -m zuikakucfd_b200.cases <generator> --n N [--seed S] --out DIR"""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__.splitlines()[0])
    ap.add_argument("generator", choices=sorted(GENERATORS))
    ap.add_argument("--n", type=int, default=256, help="cells per side (interior cells for smooth_wave)")
    ap.add_argument("--seed", type=int, default=0, help="four_quadrant: RNG seed")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    c = GENERATORS[a.generator](a)
    d = write_case(c, a.out)
    print(f"{c.name}: {c.ny}x{c.nx}, da={c.da:.6g}, gamma={c.gamma} -> {d}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
