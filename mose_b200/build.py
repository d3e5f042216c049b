"""Builds libmose_gpu.so (the C-ABI library) in-tree with nvcc for sm_100a.

The reference-exact translation unit is compiled with --fmad=false so that no
multiply-add contraction changes the rounding of the reference's FP64
expressions.  Outputs go to mose_b200/lib/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIBDIR = HERE / "lib"
OBJDIR = HERE / "_build"
LIBNAME = "libmose_gpu.so"
# measurement-only probes, linked into their own library beside the product
PROBE_DIR = HERE / "probe"
PROBE_LIB = "libmose_probe.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                 "-I", str(CSRC), "-I", str(HERE.parent / "include")]

# translation unit -> extra flags
UNITS = {
    "kernels_exact.cu": ["--fmad=false"],
    "viscous2d.cu": ["--fmad=false"],
    **{f"stage_exact_r{r}.cu": ["--fmad=false"] for r in range(5)},
    **{f"stage_fp64_r{r}.cu": [] for r in range(5)},
    **{f"stage_mixed_r{r}.cu": [] for r in range(5)},
    **{f"stage3d_exact_r{r}.cu": ["--fmad=false"] for r in (0, 1, 4)},
    **{f"stage3d_fp64_r{r}.cu": [] for r in (0, 1, 4)},
    **{f"stage3d_mixed_r{r}.cu": [] for r in (0, 1, 4)},
    "mose_gpu.cu": [],
    "norms_noalloc.cu": [],
    "fastmath_check.cu": [],
    "adjoint.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu*")) + sorted(CSRC.glob("*.h")) + [HERE.parent / "include" / "mose_gpu.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, out_dir: Path | None = None,
          defines: tuple = ()) -> Path:
    """Compiles every unit that changed and links the shared library.
    out_dir/defines build a variant elsewhere (objects and library in out_dir)."""
    global OBJDIR, LIBDIR
    if out_dir is not None:
        OBJDIR = LIBDIR = Path(out_dir)
    OBJDIR.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    extra_defs = [f"-D{d}" for d in defines]
    deps = _deps()
    objs = []
    cc = nvcc()
    jobs = []
    for unit, extra in UNITS.items():
        obj = OBJDIR / (unit + ".o")
        objs.append(obj)
        if force or _stale(obj, deps):
            jobs.append([cc] + COMMON + extra + extra_defs + ["-c", str(CSRC / unit), "-o", str(obj)])
    # units compile independently: run them in parallel
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed: " + " ".join(failed[0]))
    lib = LIBDIR / LIBNAME
    if force or _stale(lib, objs):
        cmd = [cc] + ARCH + ["-shared", "-cudart=static", "-o", str(lib)] + [str(o) for o in objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    probe = LIBDIR / PROBE_LIB
    psrc = sorted(PROBE_DIR.glob("*.cu"))
    if psrc and (force or _stale(probe, psrc)):
        cmd = [cc] + COMMON + ["-shared", "-cudart=static", "-o", str(probe)] + [str(x) for x in psrc]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
