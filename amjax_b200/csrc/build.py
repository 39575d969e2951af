"""Build libamg_b200.so (sm_100a) from the CUDA sources in this directory.

Each translation unit compiles in parallel with nvcc; objects are rebuilt only when a
source or header is newer.  Usage: ``python -m amjax_b200.csrc.build`` or
``amjax_b200.csrc.build.build()``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
OUT = PKG / "libamg_b200.so"
OBJDIR = HERE / "_build"
SOURCES = ["amg_runtime.cu", "amg_drv_f64.cu", "amg_drv_f32.cu", "amg_drv_mixed.cu", "amg_drv_mixed_cg.cu", "amg_capi.cu",
           "amg_noalloc.cu", "amg_program.cu", "amg_profile.cu"]
HEADERS = ["amg_device.cuh", "amg_runtime.cuh", "amg_pcg.cuh", "amg_drivers.cuh", "amg_program.cuh",
           str(ROOT / "include" / "amg_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newest(paths) -> float:
    return max(Path(p).stat().st_mtime for p in paths)


def build(verbose: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    OBJDIR.mkdir(exist_ok=True)
    hdr_t = _newest([HERE / h if not os.path.isabs(h) else h for h in HEADERS])
    jobs = []
    for src in SOURCES:
        obj = OBJDIR / (Path(src).stem + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(hdr_t, (HERE / src).stat().st_mtime):
            jobs.append((src, obj))

    def compile_one(job):
        src, obj = job
        cmd = [nvcc, *ARCH, *FLAGS, "-c", str(HERE / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose:
            print(f"compiled {src}", file=sys.stderr)
        return r.stderr

    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for err in ex.map(compile_one, jobs):
                if verbose and err.strip():
                    print(err, file=sys.stderr)
    objs = [OBJDIR / (Path(s).stem + ".o") for s in SOURCES]
    if force or jobs or not OUT.exists() or OUT.stat().st_mtime < _newest(objs):
        cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(OUT)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
