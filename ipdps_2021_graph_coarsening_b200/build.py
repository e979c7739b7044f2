"""In-tree build of the native libraries.

* ``libsgpar_b200.so`` -- the sm_100a kernels and the C ABI of
  ``include/sgpar_b200.h`` (``csrc/*.cu``, ``csrc/io.cpp``, ``csrc/tune.cpp``), built with nvcc
  for ``arch=compute_100a,code=sm_100a``.
* ``libsgpgen.so`` -- the synthetic graph generators (``csrc/graphgen.cpp``).
* ``sgpar_b200`` -- the config-file driver command (``csrc/sgpar_main.c``,
  the reference's ``sgpar.cpp`` main), linked against ``libsgpar_b200.so``
  with an rpath to this directory.

Objects go to ``_build/``; the libraries sit next to this file so that they
travel with the source tree.  Rebuilds are skipped when outputs are newer than
every source.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsgpar_b200.so")
GENLIB = os.path.join(HERE, "libsgpgen.so")
DRIVER = os.path.join(HERE, "sgpar_b200")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # a g++ whose OpenMP runtime spec is installed
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_lib(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(ROOT, "include", "sgpar_b200.h")]
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + [os.path.join(CSRC, "io.cpp"),
                                                             os.path.join(CSRC, "tune.cpp")]
    nvcc = _nvcc()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc] + NVCC_FLAGS + ["-c", s, "-o", o]
            if s.endswith(".cpp"):
                cmd = [nvcc, "-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-c", s, "-o", o]
            jobs.append(cmd)
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs)
    if verbose:
        print("built", LIB)
    return LIB


def build_gen(force: bool = False) -> str:
    src = os.path.join(CSRC, "graphgen.cpp")
    if force or _stale(GENLIB, [src]):
        _run([_cxx(), "-O3", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-o", GENLIB, src])
    return GENLIB


def build_driver(force: bool = False) -> str:
    src = os.path.join(CSRC, "sgpar_main.c")
    hdr = os.path.join(ROOT, "include", "sgpar_b200.h")
    if force or _stale(DRIVER, [src, hdr, LIB]):
        _run(["gcc", "-O2", "-std=c11", "-Wall", "-o", DRIVER, src, "-L" + HERE, "-lsgpar_b200",
              "-Wl,-rpath,$ORIGIN"])
    return DRIVER


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_gen(force)
    build_lib(verbose=verbose, force=force)
    build_driver(force)


if __name__ == "__main__":
    import sys
    build_all(force="--force" in sys.argv, verbose=True)
