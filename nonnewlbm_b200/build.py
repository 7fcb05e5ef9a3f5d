"""Build libnnlbm.so for sm_100a with nvcc (in-tree, next to this file).

The step kernel is compiled once per (storage type, collision) pair so that the 44
instantiations build in parallel.  FP64 units use IEEE-exact arithmetic (no fused
multiply-add contraction, no fast math) for the FP64 parity mode; the FP32-arithmetic
units use --use_fast_math like the reference's production build (solver/flags.mk:7).

    python -m nonnewlbm_b200.build [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libnnlbm.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I", str(INCLUDE),
          "--expt-relaxed-constexpr"]
F64_FLAGS = ["-fmad=false"]
F32_FLAGS = ["--use_fast_math"]
N_COLLISIONS = 11


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def units():
    """(object name, source, extra flags) for every translation unit."""
    hdrs = [CSRC / "nnlbm_kernels.cuh", CSRC / "nnlbm_physics.cuh", INCLUDE / "nnlbm.h"]
    out = [("capi", CSRC / "nnlbm_capi.cu", [], hdrs)]
    for dt in range(4):
        prec = F64_FLAGS if dt == 0 else F32_FLAGS
        out.append((f"bc_dt{dt}", CSRC / "nnlbm_bc_inst.cu", prec + [f"-DNNLBM_DT={dt}"], hdrs))
        for col in range(N_COLLISIONS):
            out.append((f"step_dt{dt}_col{col}", CSRC / "nnlbm_step_inst.cu",
                        prec + [f"-DNNLBM_DT={dt}", f"-DNNLBM_COL={col}"], hdrs))
    return out


def _stale(obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False, ptxas_info: bool = False,
          out: Path | None = None, build_dir: Path | None = None, defines=()) -> Path:
    """Compile every translation unit (skipping up-to-date objects) and link ``out``."""
    lib_path = Path(out) if out else LIB
    bdir = Path(build_dir) if build_dir else BUILD
    bdir.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    jobs = jobs or max(1, os.cpu_count() or 1)
    todo = []
    objs = []
    for name, src, extra, hdrs in units():
        obj = bdir / f"{name}.o"
        objs.append(obj)
        if force or _stale(obj, [src, *hdrs, Path(__file__)]):
            cmd = [cc, *ARCH, *COMMON, *extra, *[f"-D{d}" for d in defines], "-c", str(src), "-o", str(obj)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            todo.append((name, cmd))

    def run(item):
        name, cmd = item
        p = subprocess.run(cmd, capture_output=True, text=True)
        return name, p.returncode, p.stdout + p.stderr

    failed = []
    if todo:
        with ThreadPoolExecutor(max_workers=jobs) as ex:
            for name, rc, log in ex.map(run, todo):
                if verbose or rc != 0 or ptxas_info:
                    sys.stderr.write(f"== {name} (rc={rc})\n{log}\n")
                if rc != 0:
                    failed.append(name)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    if todo or force or not lib_path.exists() or any(o.stat().st_mtime > lib_path.stat().st_mtime for o in objs):
        tmp = lib_path.with_suffix(".so.tmp")
        cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
        subprocess.check_call(cmd)
        os.replace(tmp, lib_path)
    return lib_path


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose, ptxas_info=a.ptxas_info))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
