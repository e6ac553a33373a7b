"""Build recipes for libbgwsigma (sm_100a) and the C++11 reference shim.

Outputs (in-tree, next to the sources, so they travel with the working tree):
  lib/libbgwsigma.so          the CUDA kernels + C ABI (include/bgw_sigma.h)
  lib/libbgwsigma_check.so    the same with -DBGW_CHECK: kernels check their
                              staging ranges and tile / row / packed-buffer
                              indices and report BGW_ERR_CHECK (debug build)
  lib/libbgwsigma_refshim.so  C++11 drop-in: the reference's four kernel
                              signatures over the C ABI
  lib/bgw_refshim.o           the same shim as a PIC object, for static links

A build is skipped when a stamp of the sources and flags is unchanged.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent.parent          # berkeleygw-kernels-cpp_b200/
REPO = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
SHIM = PKG_DIR / "shim"
LIB_DIR = PKG_DIR / "lib"
INCLUDE = REPO / "include"

LIB = LIB_DIR / "libbgwsigma.so"
CHECK_LIB = LIB_DIR / "libbgwsigma_check.so"
SHIM_LIB = LIB_DIR / "libbgwsigma_refshim.so"
SHIM_OBJ = LIB_DIR / "bgw_refshim.o"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills", f"-I{INCLUDE}"]
CUDA_SOURCES = ["runtime.cu", "gpp.cu", "gpp_adjoint.cu", "gpp_batched.cu", "ff.cu", "ff_mixed.cu", "ff_fused.cu", "capi.cu", "peak.cu", "fill.cu"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libbgwsigma")
    return cand


def _stamp(paths, flags) -> str:
    h = hashlib.sha256()
    for p in sorted(paths):
        h.update(str(p.name).encode())
        h.update(p.read_bytes())
    h.update(" ".join(flags).encode())
    return h.hexdigest()


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), file=sys.stderr)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    return r


def _build_cuda_lib(lib: Path, flags, obj_dir: Path, stamp_file: Path, force: bool, verbose: bool) -> None:
    srcs = [CSRC / s for s in CUDA_SOURCES] + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "bgw_sigma.h"]
    stamp = _stamp(srcs, flags)
    if force or not lib.exists() or not stamp_file.exists() or stamp_file.read_text() != stamp:
        nvcc = _nvcc()
        objs = []
        obj_dir.mkdir(exist_ok=True)
        for s in CUDA_SOURCES:
            o = obj_dir / (Path(s).stem + ".o")
            _run([nvcc, *flags, "-c", CSRC / s, "-o", o], verbose)
            objs.append(o)
        tmp = lib.with_suffix(".so.tmp")
        _run([nvcc, *ARCH, "-shared", "-o", tmp, *objs], verbose)
        os.replace(tmp, lib)
        stamp_file.write_text(stamp)


def build_check(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the debug build libbgwsigma_check.so (-DBGW_CHECK)."""
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    _build_cuda_lib(CHECK_LIB, NVCC_FLAGS + ["-DBGW_CHECK"], LIB_DIR / "obj_check", LIB_DIR / ".check.stamp", force,
                    verbose)
    return CHECK_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles libbgwsigma.so and the shim if their sources changed."""
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    _build_cuda_lib(LIB, NVCC_FLAGS, LIB_DIR / "obj", LIB_DIR / ".libbgwsigma.stamp", force, verbose)

    shim_src = SHIM / "bgw_refshim.cpp"
    shim_stamp_file = LIB_DIR / ".refshim.stamp"
    shim_flags = ["-std=c++11", "-O2", "-fPIC", f"-I{INCLUDE}"]
    sstamp = _stamp([shim_src, INCLUDE / "bgw_sigma.h", LIB], shim_flags)
    if (force or not SHIM_LIB.exists() or not SHIM_OBJ.exists() or not shim_stamp_file.exists()
            or shim_stamp_file.read_text() != sstamp):
        _run(["g++", *shim_flags, "-c", shim_src, "-o", SHIM_OBJ], verbose)
        _run(["g++", "-shared", "-o", SHIM_LIB, SHIM_OBJ, f"-L{LIB_DIR}", "-lbgwsigma",
              "-Wl,-rpath,$ORIGIN"], verbose)
        shim_stamp_file.write_text(sstamp)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
    if "--check" in sys.argv:
        print(build_check(force="--force" in sys.argv, verbose=True))
