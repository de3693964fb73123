"""In-tree build of the native parts (no GPU needed: nvcc cross-compiles).

    python -m cudalbm_b200.build            # library + solver executables
    python -m cudalbm_b200.build --force    # rebuild everything

Outputs:
  cudalbm_b200/lib/liblbm_b200.so      C ABI of include/lbm_b200.h (sm_100a)
  cudalbm_b200/lib/liblbm_b200_checked.so  the same, its step kernels checking every index (tests)
  cudalbm_b200/bin/momentBasedD3Q19    solver executables with the reference's
  cudalbm_b200/bin/momentBasedD3Q27    command line and case files
  cudalbm_b200/bin/fieldConvert        .LBMBin -> VTS (whole fields or cut planes)
  cudalbm_b200/bin/fieldCalculate      containsNaN / spatialMean of saved times (on the GPU)
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "lib", "liblbm_b200.so")
LIB_CHECKED = os.path.join(HERE, "lib", "liblbm_b200_checked.so")  # step kernels with index checks
BIN = os.path.join(HERE, "bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-cudart", "static",
              "-I" + INCLUDE, "-I" + CSRC] + ARCH

LIB_SOURCES = ["lbm_capi.cu", "lbm_batch.cu", "lbm_closure.cu", "variants_q19_f32.cu", "variants_q27_f32.cu", "variants_f16.cu", "variants_bf16.cu",
               "lbm_noalloc.cu", "lbm_fieldcalc.cu", "casefile.cpp", "lbmbin.cpp", "postprocess.cpp"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h")))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _library_jobs(checked: bool, verbose_ptxas: bool = False):
    """(compile commands, objects, link command, output) of the library or of
    its checked build (-DLBM_CHECKED: the step kernels verify their indices)."""
    lib = LIB_CHECKED if checked else LIB
    objdir = os.path.join(HERE, "lib", "obj_checked" if checked else "obj")
    os.makedirs(objdir, exist_ok=True)
    flags = NVCC_FLAGS + (["-DLBM_CHECKED"] if checked else [])
    jobs = []
    for src in LIB_SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [_nvcc()] + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        jobs.append((cmd, obj))
    link = [_nvcc()] + flags + ["-shared"] + [o for _, o in jobs] + ["-o", lib + ".tmp"]
    return jobs, link, lib


def build_library(force: bool = False, verbose_ptxas: bool = False, checked_too: bool = True) -> str:
    """Compile every source to an object in parallel (the library and, with
    checked_too, its checked build), then link."""
    from concurrent.futures import ThreadPoolExecutor

    builds = []
    for checked in ((False, True) if checked_too else (False,)):
        lib = LIB_CHECKED if checked else LIB
        if force or _stale(lib, _deps()):
            builds.append(_library_jobs(checked, verbose_ptxas))
    if not builds:
        return LIB
    jobs = [j for b in builds for j in b[0]]
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as pool:
        list(pool.map(lambda j: _run(j[0]), jobs))
    for _, link, lib in builds:
        _run(link)
        os.replace(lib + ".tmp", lib)
    return LIB


def _cxx() -> str:
    # the system compiler (a g++ earlier on PATH may lack parts of libstdc++)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def build_executables(force: bool = False) -> list:
    """momentBasedD3Q19 / momentBasedD3Q27 and fieldCalculate (host C++ over
    the library) and fieldConvert (host only)."""
    out = []
    main = os.path.join(CSRC, "solver_main.cpp")
    os.makedirs(BIN, exist_ok=True)
    host = [os.path.join(CSRC, s) for s in ("casefile.cpp", "lbmbin.cpp")]
    for q in (19, 27):
        exe = os.path.join(BIN, f"momentBasedD3Q{q}")
        if force or _stale(exe, _deps() + [LIB]):
            _run([_cxx(), "-std=c++17", "-O2", "-Wall", "-I" + INCLUDE, "-I" + CSRC, f"-DLBM_LATTICE={q}", main] + host +
                 ["-o", exe, "-L" + os.path.dirname(LIB), "-llbm_b200", "-Wl,-rpath,$ORIGIN/../lib"])
        out.append(exe)
    # fieldCalculate: host C++ over the library (the reductions run on the GPU)
    exe = os.path.join(BIN, "fieldCalculate")
    if force or _stale(exe, _deps() + [LIB]):
        _run([_cxx(), "-std=c++17", "-O2", "-Wall", "-I" + INCLUDE, "-I" + CSRC, os.path.join(CSRC, "fieldcalculate_main.cpp")]
             + host + ["-o", exe, "-L" + os.path.dirname(LIB), "-llbm_b200", "-Wl,-rpath,$ORIGIN/../lib"])
    out.append(exe)
    # fieldConvert: host only (no GPU, no library)
    exe = os.path.join(BIN, "fieldConvert")
    srcs = [os.path.join(CSRC, s) for s in ("fieldconvert_main.cpp", "casefile.cpp", "lbmbin.cpp", "postprocess.cpp")]
    if force or _stale(exe, _deps()):
        _run([_cxx(), "-std=c++17", "-O2", "-Wall", "-I" + INCLUDE, "-I" + CSRC] + srcs + ["-o", exe])
    out.append(exe)
    return out


def build_oracle(reference_dir: str | None = None) -> None:
    """CPU oracle (test infrastructure) and, when a checkout of the reference
    is named (argument, else the LBM_REFERENCE_DIR environment variable), the
    reference executables used as the parity checker.  Without one, the
    reference binaries are not built and the tests that need them skip."""
    _run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile")])
    ref = reference_dir or os.environ.get("LBM_REFERENCE_DIR")
    if ref and os.path.isdir(os.path.join(ref, "applications")):
        _run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile.ref"), f"REF={ref}"])


def build(force: bool = False) -> None:
    build_library(force)
    build_executables(force)


if __name__ == "__main__":
    force = "--force" in sys.argv
    build(force)
    if "--oracle" in sys.argv:
        build_oracle()
