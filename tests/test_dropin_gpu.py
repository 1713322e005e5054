"""The reference's own drivers -- src_WENO/solver.cpp and src_DG/solver.cpp,
unchanged -- linked against the GPU backend (zuikakucfd_b200/adapter,
recipe `make -C oracle dropin`) write the same result files as the reference
CPU build run on the same case: the drop-in check at the level of a user who
keeps the reference's CLI."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_linf

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"


def _run(binary, case_dir, args, cwd, env=None):
    cwd.mkdir(parents=True, exist_ok=True)
    r = subprocess.run([str(binary), str(case_dir), *args], cwd=cwd, capture_output=True, text=True, timeout=600,
                       env={**os.environ, **(env or {})})
    assert r.returncode == 0, (binary.name, r.stdout[-2000:], r.stderr[-2000:])


def _result(cwd, step):
    d = cwd / "result" / str(step)
    return np.stack([np.loadtxt(d / f"U{c}_0.dat") for c in range(4)])


def _need(*names):
    missing = [n for n in names if not (REF / n).exists()]
    if missing:
        pytest.fail(f"{missing} not built: run `make -C oracle ref dropin` where the reference sources are")


def test_weno_cli_on_gpu_matches_reference_cli(tmp_path):
    from zuikakucfd_b200 import cases
    _need("solver_WENO", "dropin_WENO")
    c = cases.four_quadrant(64, seed=3)
    case = cases.write_case(c, tmp_path / "case")
    dt = f"{cases.cfl_dt(c, 0.4):.17e}"
    _run(REF / "solver_WENO", case, [dt, "100"], tmp_path / "cpu")
    _run(REF / "dropin_WENO", case, [dt, "100"], tmp_path / "gpu")
    _run(REF / "dropin_WENO", case, [dt, "100"], tmp_path / "gpu_mixed", env={"ZK_PRECISION": "mixed"})
    cpu, gpu, mixed = (_result(tmp_path / d, 100) for d in ("cpu", "gpu", "gpu_mixed"))
    assert np.isfinite(gpu).all()
    assert rel_linf(gpu, cpu) <= 1e-10
    d = np.abs(mixed[0] - gpu[0]).sum() / np.abs(gpu[0]).sum()
    assert 0 < d < 1e-5, d


@pytest.mark.parametrize("cli,P", [("DG2", 1), ("DG3", 2), ("DG4", 3)])
def test_dg_cli_on_gpu_matches_reference_cli(tmp_path, cli, P):
    """`auto` mode: the driver's own CFL check (computeMaxSpeedDG_omp, every
    10 steps) reads the modes the adapter brings back after each step."""
    from zuikakucfd_b200 import cases
    _need(f"solver_{cli}", f"dropin_{cli}")
    c = cases.four_quadrant(40, seed=4)
    case = cases.write_case(c, tmp_path / "case")
    _run(REF / f"solver_{cli}", case, ["auto", "25"], tmp_path / "cpu")
    _run(REF / f"dropin_{cli}", case, ["auto", "25"], tmp_path / "gpu")
    cpu, gpu = _result(tmp_path / "cpu", 25), _result(tmp_path / "gpu", 25)
    assert np.isfinite(gpu).all()
    assert rel_linf(gpu, cpu) <= 1e-10, P
