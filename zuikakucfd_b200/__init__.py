"""ZuikakuCFD on B200: WENO5 / DG P=1-3 explicit 2D Euler per-step compute as
hand-written sm_100a kernels behind a C ABI (include/zuikaku.h)."""
from .fluid import (Mesh, Solver, applyLimiter, combineRankSnapshots, computeMach, computeMaxSpeed, computeRHS,
                    dg_cfl_limit, exchangeConservativeColumns, loadCheckpoint, saveCheckpoint,
                    dg_safe_dt, read_case, recoverPrimitives, run, saveMeshData, splitMeshVertically, updateMesh)
from . import cases, slab

__all__ = ["Mesh", "Solver", "applyLimiter", "combineRankSnapshots", "computeMach", "computeMaxSpeed",
           "computeRHS", "dg_cfl_limit", "loadCheckpoint", "saveCheckpoint",
           "dg_safe_dt", "exchangeConservativeColumns", "read_case", "recoverPrimitives", "run", "saveMeshData",
           "splitMeshVertically", "updateMesh", "cases", "slab"]
