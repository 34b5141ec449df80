"""Build libhermite_b200.so in-tree with nvcc for sm_100a.

    python -m hermite_b200.build            # build if sources changed
    python -m hermite_b200.build --force    # rebuild
    python -m hermite_b200.build --ptxas-v  # also print register/spill usage

The library is plain CUDA C++ with a C ABI (include/hermite_b200.h); it does
not link against torch.  Object files go to hermite_b200/_build/, the shared
library to hermite_b200/_lib/ (both git-ignored; the .so travels with the
tree).
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
BUILD = PKG / "_build"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libhermite_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-fopenmp",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE), "-I", str(CSRC)]
SOURCES = ["hb_capi.cu", "hb_predict_pot.cu", "hb_force_64.cu", "hb_force_mixed.cu", "hb_force_lanes.cu",
           "hb_noalloc.cu", "hb_integrator.cu", "hb_ensemble.cu", "hb_team.cu",
           "hb_dump.cu"]
HEADERS = ["hb_common.cuh", "hb_math.cuh", "hb_force.cuh", "hb_force_table.cuh",
           "hb_internal.h", "hb_corrector.cuh", "hb_tuning.inc"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build hermite_b200")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, extra: list[str]) -> str:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "hermite_b200.h"]
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    jobs = []
    for s in SOURCES:
        src, obj = CSRC / s, BUILD / (Path(s).stem + ".o")
        if force or ptxas_verbose or _stale(obj, [src, *headers]):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            for (src, _), log in zip(jobs, ex.map(lambda j: _compile(j[0], j[1], extra), jobs)):
                if log.strip() and (ptxas_verbose or not quiet):
                    print(f"== {src.name}\n{log}", file=sys.stderr)
    objs = [BUILD / (Path(s).stem + ".o") for s in SOURCES]
    if force or jobs or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-cudart", "static",
               "-Xcompiler", "-fopenmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_v, quiet=False))


if __name__ == "__main__":
    main()
