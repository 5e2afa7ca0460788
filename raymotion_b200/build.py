"""Build recipe of the native library, ``raymotion_b200/librmcuda.so``.

Every CUDA translation unit is compiled ahead of time for sm_100a with nvcc
(no JIT, no torch extension cache): the library is built in the source tree
so that it travels with it.  ``-fmad=false`` keeps every a*b+c unfused and the
default ``-prec-div=true -prec-sqrt=true -ftz=false`` keep division, square
root and denormals IEEE-exact: on identical RNG streams the kernels then
reproduce the CPU oracle's fp32 radiance bit for bit.
"""
from __future__ import annotations

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
LIB = PKG / "librmcuda.so"
# The checked build: the same sources with RMCUDA_CHECKED defined (device-side
# bounds checks that set an error bit and skip the access, see rm_device.cuh);
# loaded instead of LIB when RAYMOTION_CUDA_CHECKED=1.
BUILD_CHECKED = PKG / "_build_checked"
LIB_CHECKED = PKG / "librmcuda_checked.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-fmad=false",
    "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    f"-I{ROOT / 'include'}", f"-I{CSRC}",
]
CU_SOURCES = ["rm_kernels.cu", "rm_denoise.cu", "rm_bvh.cu", "rmcuda_api.cu", "rm_noalloc.cu", "rm_wavefront.cu",
              "rm_atrous.cu", "rm_batch.cu", "rmcuda_batch.cu", "rm_adjoint.cu", "rm_denoise_adjoint.cu",
              "rmcuda_adjoint.cu", "rm_wide.cu", "rm_prep.cu", "rm_sort.cu"]
# Tolerance-checked kernels (approximate exp2 / rsqrt anyway) are compiled with FMA contraction.
FMA_SOURCES = {"rm_atrous.cu"}
CXX_SOURCES = ["shim_metal.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}")


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose: bool = False, ptxas_info: bool = False, checked: bool = False) -> Path:
    """Compile every source and link ``librmcuda.so`` (``checked``: the bounds-checked
    ``librmcuda_checked.so``); returns its path."""
    nvcc = _nvcc()
    build_dir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    build_dir.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").rglob("*.h*"))
    jobs = []
    objs = []
    for src in CU_SOURCES + CXX_SOURCES:
        s = CSRC / src
        o = build_dir / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if (ptxas_info and src.endswith(".cu")) else []
            lang = [] if src.endswith(".cu") else ["-x", "c++"]
            flags = [f for f in NVFLAGS if not (src in FMA_SOURCES and f == "-fmad=false")]
            if src in FMA_SOURCES:
                flags.append("-fmad=true")
            if checked:
                flags.append("-DRMCUDA_CHECKED")
            jobs.append([nvcc, *flags, *extra, *lang, "-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for cmd, fut in [(c, ex.submit(_run, c)) for c in jobs]:
            fut.result()
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
    if jobs or not lib.exists():
        tmp = lib.with_suffix(".so.tmp")
        _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"])
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv, checked="--checked" in sys.argv))
