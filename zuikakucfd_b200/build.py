"""Build the native library zuikakucfd_b200/lib/libzuikaku.so for sm_100a.

    python -m zuikakucfd_b200.build [--force] [-v]

Each CUDA source is compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
with its own flags (the FP64 reference-arithmetic kernels use ``--fmad=false``
so that every multiply and add rounds separately, as the reference does when
built with -ffp-contract=off), then all objects are linked into one shared
library with the CUDA runtime linked statically, so the library loads through
ctypes without any Python CUDA stack.  Objects go to ``_build/`` next to this
file; the build is incremental on file times.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libzuikaku.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          f"-I{CSRC}", f"-I{ROOT / 'include'}", "--expt-relaxed-constexpr"]
STRICT = ["--fmad=false"]

# FP64 with fused multiply-add contraction: the same FP64 sources compiled a
# second time into namespace zk_fma (ZK_PREC_FP64_FMA)
FMA = ["-DZK_FP64_FMA"]

# (source, extra flags[, object name])
SOURCES: list[tuple] = [
    ("zk_api.cu", []),
    ("weno_fp64.cu", STRICT),
    ("weno_fp64.cu", FMA, "weno_fp64_fma.o"),
    ("reduce_fp64.cu", STRICT),
    ("dg_fp64.cu", STRICT),
    ("dg_fp64.cu", FMA, "dg_fp64_fma.o"),
    ("dg_driver.cu", []),
    ("dg_mixed.cu", ["--use_fast_math"]),
    ("dg_fused_fp64.cu", []),
    ("dg_tvb.cu", STRICT),
    ("mlp.cu", []),
    ("peak.cu", []),
    ("weno_mixed.cu", ["--use_fast_math"]),
    ("noalloc.cu", []),
    ("slab.cu", []),
    ("batch.cu", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the native library needs the CUDA toolkit")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps, Path(__file__)])


def _compile(src: Path, flags: list[str], force: bool, verbose: bool, obj_name: str | None = None) -> Path:
    obj = OBJ / (obj_name or src.stem + ".o")
    if not force and not _stale(obj, src, _headers()):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda sf: _compile(CSRC / sf[0], sf[1], force, verbose, *sf[2:]), SOURCES))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print nvcc lines and -Xptxas -v")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
