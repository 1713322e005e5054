"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two back ends with the same methods:

* ``Restatement`` -- oracle/_build/liboracle.so, the project's own C
  restatement of the reference hot path (weno_oracle.c, dg_oracle.c);
* ``Reference``   -- oracle/_ref/libref_*.so, the reference's own sources
  compiled unmodified against oracle/shim (see oracle/Makefile), in the
  variants "faithful" (the reference Makefile's flags, FMA contraction on),
  "strict" (-ffp-contract=off) and "omp" (faithful + -fopenmp).

Only tests/, __graft_entry__.smoke() and the CPU-baseline legs of bench.py use
this module, as the checker of the GPU path.  Arrays are row-major:
U[4][ny][nx], dof[4][NM][ny][nx], bctype int32[ny][nx].
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
# Where the reference checkout lies: ZK_REFERENCE_DIR, else the read-only
# checkout this build was made against.  Only build() and the golden-vector
# generator read it; built outputs go to _ref/ and travel without it.
REFERENCE_SOURCES = Path(os.environ.get("ZK_REFERENCE_DIR", "/root/reference"))
RESTATEMENT = HERE / "_build" / "liboracle.so"

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _i(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def build(reference: bool = True) -> None:
    """Compile the restatement and, when the reference sources exist, oracle/_ref
    (with the drop-in CLIs once the native library is built)."""
    targets = ["restatement"]
    if reference and (REFERENCE_SOURCES / "src_WENO" / "fluid.cpp").exists():
        targets.append("ref")
        lib = HERE.parent / "zuikakucfd_b200" / "lib" / "libzuikaku.so"
        if lib.exists():  # the reference CLIs linked against the GPU backend
            targets.append("dropin")
    subprocess.run(["make", "-s", "-C", str(HERE), "-j8", f"REF={REFERENCE_SOURCES}", *targets], check=True)


def host_has_avx512() -> bool:
    """The host CPU implements the x86-64-v4 level (AVX-512 F/BW/CD/DQ/VL)."""
    try:
        flags = next(l for l in Path("/proc/cpuinfo").read_text().splitlines() if l.startswith("flags")).split()
    except (OSError, StopIteration):
        return False
    return all(f in flags for f in ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"))


def reference_available(variant: str = "faithful") -> bool:
    suffix = {"faithful": "", "strict": "_strict", "omp": "_omp"}[variant]
    return (REF_DIR / f"libref_weno{suffix}.so").exists()


class Restatement:
    """The project's C restatement (bit-identical to the strict reference build)."""

    def __init__(self):
        if not RESTATEMENT.exists():
            raise RuntimeError(f"{RESTATEMENT} missing: run `make -C oracle restatement`")
        L = C.CDLL(str(RESTATEMENT))
        L.ow_rhs.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int, _D]
        L.ow_step.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int, C.c_int]
        L.ow_step_recon.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int, C.c_int,
                                    C.c_int]
        L.ow_muscl.argtypes = [C.c_double] * 4 + [C.c_int, _D, _D]
        L.ow_max_speed.argtypes = [C.c_int, C.c_int, C.c_double, _D]
        L.ow_max_speed.restype = C.c_double
        L.ow_recover.argtypes = [C.c_int, C.c_int, C.c_double, _D, _D]
        L.ow_hllc.argtypes = [_D, _D, C.c_double, _D]
        L.ow_weno5.argtypes = [C.c_double] * 6 + [_D, _D]
        L.ow_ghost_map.argtypes = [C.c_int, C.c_int, _I, C.c_int, C.c_int, C.POINTER(C.c_int8), _I]
        L.od_rhs.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_int, C.c_int, _D]
        L.od_limit.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _D, _I]
        L.od_step.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double,
                              C.c_int, C.c_int, C.c_int]
        L.od_max_speed.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _D, _I]
        L.od_max_speed.restype = C.c_double
        L.od_safe_dt.argtypes = [C.c_int, C.c_double, C.c_double]
        L.od_safe_dt.restype = C.c_double
        L.od_hllc.argtypes = [_D, _D, C.c_double, _D]
        L.od_hlle.argtypes = [_D, _D, C.c_double, _D]
        L.od_phi2.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
        L.od_phi2.restype = C.c_double
        L.od_euler_eigen.argtypes = [_D, C.c_double, C.c_int, _D, _D]
        L.od_limit_tvb.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double,
                                   C.c_int, C.POINTER(C.c_uint8)]
        L.od_step_lim.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double,
                                  C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
        self.L = L

    # WENO -----------------------------------------------------------------------
    def weno_rhs(self, U, bct, da, gamma, dt, periodic=False):
        U = np.array(U, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        dU = np.empty_like(U)
        ny, nx = b.shape
        self.L.ow_rhs(ny, nx, da, gamma, _d(U), _i(b), dt, int(periodic), _d(dU))
        return U, dU

    def weno_step(self, U, bct, da, gamma, dt, nsteps=1, periodic=False, recon=0):
        """recon 0: WENO5 (the reference path); 1..3: MUSCL with minmod, van
        Leer, superbee (the reference's muscl_reconstruct as the face
        reconstruction)."""
        U = np.array(U, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        ny, nx = b.shape
        self.L.ow_step_recon(ny, nx, da, gamma, _d(U), _i(b), dt, int(nsteps), int(periodic), int(recon))
        return U

    def muscl(self, stencils, limiter):
        """ow_muscl over stencils[n][4] = (UL2, UL1, UR1, UR2): out[n][2] = (UL, UR)."""
        st = np.ascontiguousarray(stencils, np.float64)
        out = np.empty((len(st), 2))
        ul, ur = C.c_double(), C.c_double()
        for i, (a, b, c, d) in enumerate(st):
            self.L.ow_muscl(a, b, c, d, int(limiter), C.byref(ul), C.byref(ur))
            out[i] = ul.value, ur.value
        return out

    def weno_max_speed(self, U, gamma):
        U = np.ascontiguousarray(U, dtype=np.float64)
        return self.L.ow_max_speed(U.shape[1], U.shape[2], gamma, _d(U))

    def weno_recover(self, U, gamma):
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = np.empty_like(U)
        self.L.ow_recover(U.shape[1], U.shape[2], gamma, _d(U), _d(out))
        return out

    def hllc_weno(self, L, R, gamma):
        L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
        F = np.empty(4)
        self.L.ow_hllc(_d(L), _d(R), gamma, _d(F))
        return F

    def weno5(self, *v):
        ul, ur = C.c_double(), C.c_double()
        self.L.ow_weno5(*[float(x) for x in v], C.byref(ul), C.byref(ur))
        return ul.value, ur.value

    def ghost_map(self, bct, with_slip=False, periodic=False):
        b = np.ascontiguousarray(bct, dtype=np.int32)
        kind = np.empty(b.shape, np.int8)
        src = np.empty(b.shape, np.int32)
        self.L.ow_ghost_map(b.shape[0], b.shape[1], _i(b), int(with_slip), int(periodic),
                            kind.ctypes.data_as(C.POINTER(C.c_int8)), _i(src))
        return kind, src

    # DG -------------------------------------------------------------------------
    def dg_rhs(self, P, dof, bct, da, gamma, periodic=False, hll=False):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        dU = np.empty_like(d)
        ny, nx = b.shape
        rc = self.L.od_rhs(P, ny, nx, da, gamma, _d(d), _i(b), int(periodic), int(hll), _d(dU))
        assert rc == 0
        return d, dU

    def dg_limit(self, P, dof, bct, gamma):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        self.L.od_limit(P, b.shape[0], b.shape[1], gamma, _d(d), _i(b))
        return d

    def dg_step(self, P, dof, bct, da, gamma, dt, nsteps=1, periodic=False, hll=False):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        rc = self.L.od_step(P, b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), dt, int(nsteps),
                            int(periodic), int(hll))
        assert rc == 0
        return d

    def euler_eigen(self, u, gamma, direction):
        u = np.ascontiguousarray(u, np.float64)
        L = np.zeros((4, 4)); R = np.zeros((4, 4))
        ok = self.L.od_euler_eigen(_d(u), gamma, direction, _d(L), _d(R))
        return bool(ok), L, R

    def dg_limit_tvb(self, P, dof, bct, da, gamma, M=50.0, periodic=False):
        """One TVB pass; returns (limited dof, troubled-cell flags)."""
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        fl = np.zeros(b.shape, np.uint8)
        self.L.od_limit_tvb(P, b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), M, int(periodic),
                            fl.ctypes.data_as(C.POINTER(C.c_uint8)))
        return d, fl

    def dg_step_lim(self, P, dof, bct, da, gamma, dt, nsteps=1, limiter="tvb", M=50.0, periodic=False, hll=False):
        code = {"reference": 0, "none": 1, "tvb": 2}[limiter]
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        rc = self.L.od_step_lim(P, b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), dt, int(nsteps),
                                int(periodic), int(hll), code, M)
        assert rc == 0
        return d

    def dg_max_speed(self, P, dof, bct, gamma):
        d = np.ascontiguousarray(dof, dtype=np.float64)
        b = np.ascontiguousarray(bct, dtype=np.int32)
        return self.L.od_max_speed(P, b.shape[0], b.shape[1], gamma, _d(d), _i(b))

    def dg_safe_dt(self, P, lam, h):
        return self.L.od_safe_dt(P, lam, h)

    def hllc_dg(self, L, R, gamma):
        L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
        F = np.empty(4)
        self.L.od_hllc(_d(L), _d(R), gamma, _d(F))
        return F

    def hlle_dg(self, L, R, gamma):
        L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
        F = np.empty(4)
        self.L.od_hlle(_d(L), _d(R), gamma, _d(F))
        return F

    def phi2(self, P, m, xi, eta):
        return self.L.od_phi2(P, m, xi, eta)


class Reference:
    """The unmodified reference sources (oracle/_ref), single rank."""

    def __init__(self, variant: str = "faithful"):
        self.suffix = {"faithful": "", "strict": "_strict", "omp": "_omp"}[variant]
        self.variant = variant
        self.isa = "x86-64-v3"
        # the faithful build closest to the reference Makefile's -march=native:
        # AVX-512 where the host has it
        if variant == "faithful" and host_has_avx512() and (REF_DIR / "libref_weno_v4.so").exists():
            self.suffix, self.isa = "_v4", "x86-64-v4"
        self._weno = None
        self._dg: dict[int, C.CDLL] = {}

    def _w(self):
        if self._weno is None:
            p = REF_DIR / f"libref_weno{self.suffix}.so"
            if not p.exists():
                raise RuntimeError(f"{p} missing: run `make -C oracle ref` where the reference is present")
            L = C.CDLL(str(p))
            L.refw_rhs.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, _D]
            L.refw_step.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int, C.c_int]
            L.refw_step_timed.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int]
            L.refw_step_timed.restype = C.c_double
            L.refw_max_speed.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I]
            L.refw_max_speed.restype = C.c_double
            L.refw_recover.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, _D]
            L.refw_hllc.argtypes = [_D, _D, C.c_double, _D]
            L.refw_muscl.argtypes = [_D, C.c_int, C.c_int, _D]
            L.refw_case_info.argtypes = [C.c_char_p, _I, _I, _D, _D]
            L.refw_load_case.argtypes = [C.c_char_p, _D, _I]
            L.refw_step_slabs_timed.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double,
                                                C.c_int, C.c_int, C.POINTER(C.c_long)]
            L.refw_step_slabs_timed.restype = C.c_double
            self._weno = L
        return self._weno

    def _g(self, P: int):
        if P not in self._dg:
            p = REF_DIR / f"libref_dg{P}{self.suffix}.so"
            if not p.exists():
                raise RuntimeError(f"{p} missing: run `make -C oracle ref` where the reference is present")
            L = C.CDLL(str(p))
            L.refd_rhs.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, _D]
            L.refd_limit.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I]
            L.refd_step.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int, C.c_int]
            L.refd_step_timed.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double, C.c_int]
            L.refd_step_timed.restype = C.c_double
            L.refd_max_speed.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I]
            L.refd_max_speed.restype = C.c_double
            L.refd_safe_dt.argtypes = [C.c_double, C.c_double]
            L.refd_safe_dt.restype = C.c_double
            L.refd_hllc.argtypes = [_D, _D, C.c_double, _D]
            L.refd_hlle.argtypes = [_D, _D, C.c_double, _D]
            L.refd_phi2.argtypes = [C.c_int, C.c_double, C.c_double]
            L.refd_phi2.restype = C.c_double
            L.refd_case_info.argtypes = [C.c_char_p, _I, _I, _D, _D]
            L.refd_load_case.argtypes = [C.c_char_p, _D, _I]
            L.refd_step_slabs_timed.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D, _I, C.c_double,
                                                C.c_int, C.c_int, C.POINTER(C.c_long)]
            L.refd_step_slabs_timed.restype = C.c_double
            assert L.refd_order() == P
            self._dg[P] = L
        return self._dg[P]

    # WENO -----------------------------------------------------------------------
    def weno_rhs(self, U, bct, da, gamma, dt):
        U = np.array(U, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        dU = np.empty_like(U)
        self._w().refw_rhs(b.shape[0], b.shape[1], da, gamma, _d(U), _i(b), dt, _d(dU))
        return U, dU

    def weno_step(self, U, bct, da, gamma, dt, nsteps=1, periodic=False):
        U = np.array(U, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        self._w().refw_step(b.shape[0], b.shape[1], da, gamma, _d(U), _i(b), dt, int(nsteps), int(periodic))
        return U

    def weno_step_timed(self, U, bct, da, gamma, dt, nsteps=1):
        U = np.array(U, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        ms = self._w().refw_step_timed(b.shape[0], b.shape[1], da, gamma, _d(U), _i(b), dt, int(nsteps))
        return U, ms

    def weno_slabs_timed(self, U, bct, da, gamma, dt, nsteps, nthreads):
        """(ms of the slowest slab, updated cells) for nthreads x-slabs run
        concurrently (timing emulation of an MPI run; see the harness)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        b = np.ascontiguousarray(bct, dtype=np.int32)
        cells = C.c_long()
        ms = self._w().refw_step_slabs_timed(b.shape[0], b.shape[1], da, gamma, _d(U), _i(b), dt,
                                            int(nsteps), int(nthreads), C.byref(cells))
        return ms, cells.value

    def weno_max_speed(self, U, bct, da, gamma):
        U = np.ascontiguousarray(U, dtype=np.float64)
        b = np.ascontiguousarray(bct, dtype=np.int32)
        return self._w().refw_max_speed(b.shape[0], b.shape[1], da, gamma, _d(U), _i(b))

    def weno_recover(self, U, bct, da, gamma):
        U = np.ascontiguousarray(U, dtype=np.float64)
        b = np.ascontiguousarray(bct, dtype=np.int32)
        out = np.empty_like(U)
        self._w().refw_recover(b.shape[0], b.shape[1], da, gamma, _d(U), _i(b), _d(out))
        return out

    def hllc_weno(self, L, R, gamma):
        L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
        F = np.empty(4)
        self._w().refw_hllc(_d(L), _d(R), gamma, _d(F))
        return F

    def muscl(self, stencils, limiter):
        """The reference's muscl_reconstruct over stencils[n][4]: out[n][2] = (UL, UR)."""
        st = np.ascontiguousarray(stencils, np.float64)
        out = np.empty((len(st), 2))
        self._w().refw_muscl(_d(st), len(st), int(limiter), _d(out))
        return out

    def weno_load_case(self, folder):
        ny, nx = C.c_int(), C.c_int()
        da, g = C.c_double(), C.c_double()
        assert self._w().refw_case_info(str(folder).encode(), C.byref(ny), C.byref(nx), C.byref(da), C.byref(g)) == 0
        U = np.empty((4, ny.value, nx.value))
        b = np.empty((ny.value, nx.value), np.int32)
        assert self._w().refw_load_case(str(folder).encode(), _d(U), _i(b)) == 0
        return U, b, da.value, g.value

    # DG -------------------------------------------------------------------------
    def dg_rhs(self, P, dof, bct, da, gamma, dt=0.0):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        dU = np.empty_like(d)
        self._g(P).refd_rhs(b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), dt, _d(dU))
        return d, dU

    def dg_limit(self, P, dof, bct, da, gamma):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        self._g(P).refd_limit(b.shape[0], b.shape[1], da, gamma, _d(d), _i(b))
        return d

    def dg_step(self, P, dof, bct, da, gamma, dt, nsteps=1, periodic=False):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        self._g(P).refd_step(b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), dt, int(nsteps), int(periodic))
        return d

    def dg_step_timed(self, P, dof, bct, da, gamma, dt, nsteps=1):
        d = np.array(dof, dtype=np.float64, order="C")
        b = np.ascontiguousarray(bct, dtype=np.int32)
        ms = self._g(P).refd_step_timed(b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), dt, int(nsteps))
        return d, ms

    def dg_slabs_timed(self, P, dof, bct, da, gamma, dt, nsteps, nthreads):
        d = np.ascontiguousarray(dof, dtype=np.float64)
        b = np.ascontiguousarray(bct, dtype=np.int32)
        cells = C.c_long()
        ms = self._g(P).refd_step_slabs_timed(b.shape[0], b.shape[1], da, gamma, _d(d), _i(b), dt,
                                              int(nsteps), int(nthreads), C.byref(cells))
        return ms, cells.value

    def dg_max_speed(self, P, dof, bct, da, gamma):
        d = np.ascontiguousarray(dof, dtype=np.float64)
        b = np.ascontiguousarray(bct, dtype=np.int32)
        return self._g(P).refd_max_speed(b.shape[0], b.shape[1], da, gamma, _d(d), _i(b))

    def dg_safe_dt(self, P, lam, h):
        return self._g(P).refd_safe_dt(lam, h)

    def hllc_dg(self, L, R, gamma, P=2):
        L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
        F = np.empty(4)
        self._g(P).refd_hllc(_d(L), _d(R), gamma, _d(F))
        return F

    def hlle_dg(self, L, R, gamma, P=2):
        L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
        F = np.empty(4)
        self._g(P).refd_hlle(_d(L), _d(R), gamma, _d(F))
        return F

    def phi2(self, P, m, xi, eta):
        return self._g(P).refd_phi2(m, xi, eta)
