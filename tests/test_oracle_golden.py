"""The CPU oracle (the project's C restatement) against golden vectors
produced by RUNNING the reference's own sources (tests/golden/gen_golden.py).

"strict" goldens come from the reference built with -ffp-contract=off: the
restatement must match them bit for bit.  "faithful" goldens come from the
reference Makefile's flags (FMA contraction): within 1e-10 relative L-inf.
"""
import hashlib

import numpy as np
import pytest

from conftest import rel_linf

WENO = ["weno_fq_24x24_s3", "weno_fq_23x37_s11", "weno_fq_7x7_s5", "weno_obstacle_26",
        "weno_jet_40x20", "weno_allghost_12"]
DG = [f"dg{P}_{c}" for P in (1, 2, 3) for c in ("fq20", "fq17x23", "slip22", "vacuum18")]


@pytest.mark.parametrize("name", WENO)
def test_weno_steps_bit_exact(restatement, golden, golden_meta, name):
    m = golden_meta[name]
    U0, b = golden[f"{name}/U0"], golden[f"{name}/bct"]
    for n in m["steps"]:
        out = restatement.weno_step(U0, b, m["da"], m["gamma"], m["dt"], n)
        assert np.array_equal(out, golden[f"{name}/strict_{n}"]), (name, n)
        assert rel_linf(out, golden[f"{name}/faithful_{n}"]) < 1e-10


@pytest.mark.parametrize("name", WENO)
def test_weno_rhs_fill_speed_recover(restatement, golden, golden_meta, name):
    m = golden_meta[name]
    U0, b = golden[f"{name}/U0"], golden[f"{name}/bct"]
    Uf, dU = restatement.weno_rhs(U0, b, m["da"], m["gamma"], m["dt"])
    assert np.array_equal(Uf, golden[f"{name}/rhs_U"])      # ghost fill, in place
    assert np.array_equal(dU, golden[f"{name}/rhs_dU"])
    assert restatement.weno_max_speed(U0, m["gamma"]) == m["max_speed"]
    S = golden[f"{name}/strict_10"]
    assert restatement.weno_max_speed(S, m["gamma"]) == m["max_speed_10"]
    assert np.array_equal(restatement.weno_recover(S, m["gamma"]), golden[f"{name}/prim_10"], equal_nan=True)


def test_weno_periodic_wave(restatement, golden, golden_meta):
    m = golden_meta["weno_wave_16"]
    out = restatement.weno_step(golden["weno_wave_16/U0"], golden["weno_wave_16/bct"], m["da"],
                                m["gamma"], m["dt"], 5, periodic=True)
    assert np.array_equal(out, golden["weno_wave_16/strict_5"])
    assert rel_linf(out, golden["weno_wave_16/faithful_5"]) < 1e-10


def test_weno_reference_riemann_case_hash(restatement, golden, golden_meta):
    """The reference's own 2D-Riemann input (256x256): 20 steps, SHA-256 of the
    strict reference result."""
    m = golden_meta["riemann256"]
    U, b, g = golden["riemann256/U0"], golden["riemann256/bct"], m["gamma"]
    assert restatement.weno_max_speed(U, g) == m["max_speed"]
    out = restatement.weno_step(U, b, m["da"], g, m["dt"], m["steps"])
    assert hashlib.sha256(out.tobytes()).hexdigest() == m["strict_sha256"]
    assert np.array_equal(out[:, ::17], golden["riemann256/strict_20_rows"])
    assert rel_linf(out[:, ::17], golden["riemann256/faithful_20_rows"]) < 1e-10


@pytest.mark.parametrize("name", DG)
def test_dg_steps_bit_exact(restatement, golden, golden_meta, name):
    m = golden_meta[name]
    P = m["P"]
    d0, b = golden[f"{name}/dof0"], golden[f"{name}/bct"]
    out = restatement.dg_step(P, d0, b, m["da"], m["gamma"], m["dt"], 3)
    ref = golden[f"{name}/strict_3"]
    # log10/sin in the Persson filter come from libm on both sides: bit-exact
    # on the same host, 1e-12 elsewhere
    assert rel_linf(out, ref) <= 1e-12, name
    assert rel_linf(out, golden[f"{name}/faithful_3"]) < 1e-10


@pytest.mark.parametrize("name", DG)
def test_dg_rhs_limit_speed(restatement, golden, golden_meta, name):
    m = golden_meta[name]
    P = m["P"]
    d0, b = golden[f"{name}/dof0"], golden[f"{name}/bct"]
    x, dU = restatement.dg_rhs(P, d0, b, m["da"], m["gamma"])
    assert np.array_equal(x, golden[f"{name}/rhs_dof"])
    assert np.array_equal(dU, golden[f"{name}/rhs_dU"])
    lim = restatement.dg_limit(P, d0, b, m["gamma"])
    assert rel_linf(lim, golden[f"{name}/limit"]) <= 1e-12
    assert restatement.dg_max_speed(P, d0, b, m["gamma"]) == m["max_speed"]


@pytest.mark.parametrize("P", [1, 2, 3])
def test_dg_periodic_wave(restatement, golden, golden_meta, P):
    name = f"dg{P}_wave12"
    m = golden_meta[name]
    out = restatement.dg_step(P, golden[f"{name}/dof0"], golden[f"{name}/bct"], m["da"], m["gamma"],
                              m["dt"], 3, periodic=True)
    assert rel_linf(out, golden[f"{name}/strict_3"]) <= 1e-12
    assert rel_linf(out, golden[f"{name}/faithful_3"]) < 1e-10


def test_limiter_goldens_exercise_both_stages(golden):
    """The vacuum cases must actually trigger Zhang-Shu (modes scaled) so the
    limiter goldens test something."""
    for P in (1, 2, 3):
        d0 = golden[f"dg{P}_vacuum18/dof0"]
        lim = golden[f"dg{P}_vacuum18/limit"]
        assert not np.array_equal(d0[:, 1:], lim[:, 1:])


def test_riemann_point_vectors(restatement, golden):
    L, R = golden["points/L"], golden["points/R"]
    g = 1.4
    for k in range(L.shape[0]):
        np.testing.assert_array_equal(restatement.hllc_weno(L[k], R[k], g), golden["points/hllc_weno"][k])
        np.testing.assert_array_equal(restatement.hllc_dg(L[k], R[k], g), golden["points/hllc_dg"][k])
        np.testing.assert_array_equal(restatement.hlle_dg(L[k], R[k], g), golden["points/hlle_dg"][k])
    pts = golden["points/phi2_pts"]
    for P in (1, 2, 3):
        tab = golden[f"points/phi2_P{P}"]
        for m in range(tab.shape[0]):
            for a, xa in enumerate(pts):
                for c, xb in enumerate(pts):
                    assert restatement.phi2(P, m, xa, xb) == tab[m, a, c]


def test_ghost_map_last_writer_rule(restatement):
    """Row sweep then column sweep, last writer wins (src_WENO/fluid.cpp:338-370):
    top ghost rows 0,1,2 take interior rows 3,4,5's... of the column sweep
    where a column source exists; corners stay unfilled."""
    b = np.zeros((12, 12), np.int32)
    b[:3] = b[-3:] = -1
    b[:, :3] = b[:, -3:] = -1
    kind, src = restatement.ghost_map(b)
    nx = 12
    # left ghost column 0 in an interior row: column sweep, last writer is the
    # largest source column within 3 -> column 3 (only j=3 is within reach of 0)
    assert src[5, 0] == 5 * nx + 3
    assert src[5, 2] == 5 * nx + 5   # 2 is reached from 3, 4, 5 -> 5 wins
    assert src[5, 11] == 5 * nx + 8  # right ghosts: only columns 8 within reach of 11
    assert src[5, 9] == 5 * nx + 8   # 9 is reached from 6, 7, 8 -> 8 wins
    assert src[0, 5] == 3 * nx + 5   # top: row sweep, only row 3 reaches row 0
    assert src[2, 5] == 5 * nx + 5   # row 2 reached from 3, 4, 5 -> 5 wins
    assert src[10, 5] == 8 * nx + 5
    assert src[0, 0] == -1 and kind[0, 0] == 1  # corner never filled


def test_muscl_point_vectors(restatement, golden):
    """MUSCL reconstruction (the reference's muscl_reconstruct, dead code in
    its solvers and an option here): the restatement equals the strict
    reference build bit for bit, and the Makefile-faithful build too."""
    st = golden["muscl/stencils"]
    for lim in (0, 1, 2):
        out = restatement.muscl(st, lim)
        np.testing.assert_array_equal(out, golden[f"muscl/strict_L{lim}"])
        np.testing.assert_array_equal(out, golden[f"muscl/faithful_L{lim}"])
