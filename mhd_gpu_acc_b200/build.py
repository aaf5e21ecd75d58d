"""In-tree build of libmhd_b200.so for sm_100a (nvcc cross-compiles without a GPU).

Per-file flags matter for numerics:
  step_f64.cu   --fmad=false      FP64 step, bit-exact with the reference CPU path
  step_f32.cu   --use_fast_math   FP32-bulk step
Everything else uses the defaults.  The CUDA runtime is linked statically so the
library only needs the driver at run time.

Usage: python -m mhd_gpu_acc_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmhd_b200.so")
DRIVER = os.path.join(PKG, "mhd_run_case")  # the init / step / output driver (csrc/driver.cpp)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
               "-I", os.path.join(ROOT, "include")] + ARCH
CU_SOURCES = {
    "step_f64.cu": ["--fmad=false"],
    "step_f32.cu": ["--use_fast_math"],
    "aux_kernels.cu": [],
    "capi.cu": [],
    "noalloc.cu": [],
    "state_io.cu": [],
    "compat.cu": ["--fmad=false"],
    "ic_kernels.cu": ["--fmad=false"],
    "batch_api.cu": [],
    "adjoint.cu": [],
}
CXX_SOURCES = {"cases.cpp": []}
HEADERS = [f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] if os.path.isdir(CSRC) else []


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "mhd_b200.h")]
    for d, _, files in os.walk(os.path.join(ROOT, "include", "mhd_b200")):
        hdrs += [os.path.join(d, f) for f in files]
    tasks, objs = [], []
    nv = nvcc()
    for src, flags in CU_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            tasks.append([nv, *NVCC_COMMON, *flags, "-c", s, "-o", o])
    for src, flags in CXX_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            tasks.append(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I",
                          os.path.join(ROOT, "include"), *flags, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for cmd in tasks:
            if verbose:
                print(" ".join(cmd))
        list(ex.map(_run, tasks))
    if tasks or force or _stale(LIB, objs):
        _run([nv, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs, "-lpthread", "-ldl", "-lrt"])
    drv_src = os.path.join(CSRC, "driver.cpp")
    if force or _stale(DRIVER, [drv_src, LIB] + hdrs):
        _run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), drv_src, "-o", DRIVER, "-L", PKG,
              "-lmhd_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.j, verbose=a.v))
    return 0


if __name__ == "__main__":
    sys.exit(main())
