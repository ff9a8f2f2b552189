"""Build the sm_100a shared library in-tree: lbfast_b200/_lib/liblbfast_b200.so.

Every CUDA source is compiled with nvcc for ``-gencode arch=compute_100a,code=sm_100a``
(no other architecture), in parallel, then linked with the host C++ sources.
Rebuilds only what changed (sources newer than their objects, or any header
newer than every object).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "liblbfast_b200.so")
DRIVER = os.path.join(LIBDIR, "lbfast")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
           "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # the system g++ (an exported CXX may point at a reduced toolchain)
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _stale(src: str, obj: str, headers: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    if os.path.getmtime(src) > t:
        return True
    return any(os.path.getmtime(h) > t for h in headers)


def _compile(cmd: list[str], log: str) -> tuple[int, str]:
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.returncode, r.stdout + r.stderr


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(f for f in glob.glob(os.path.join(CSRC, "*.cpp")) if not f.endswith("lbfast_main.cpp"))
    jobs_list = []
    objs = []
    for src in cu:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(src, obj, headers):
            jobs_list.append(([nvcc, *ARCH, *NVFLAGS, "-c", src, "-o", obj], obj + ".log"))
    for src in cpp:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(src, obj, headers):
            jobs_list.append(([_host_cxx(), "-O2", "-fPIC", "-std=c++17", f"-I{INCLUDE}", "-c", src, "-o", obj],
                              obj + ".log"))
    if jobs_list:
        n = jobs or min(len(jobs_list), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(n) as ex:
            results = list(ex.map(lambda a: _compile(*a), jobs_list))
        for (cmd, log), (rc, out) in zip(jobs_list, results):
            if verbose:
                print(out)
            if rc != 0:
                raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{out}")
    if jobs_list or not os.path.exists(LIB):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}{r.stderr}")
    main = os.path.join(CSRC, "lbfast_main.cpp")
    if os.path.exists(main) and (not os.path.exists(DRIVER) or os.path.getmtime(main) > os.path.getmtime(DRIVER)
                                 or os.path.getmtime(LIB) > os.path.getmtime(DRIVER)):
        cmd = [_host_cxx(), "-O2", "-std=c++17", f"-I{INCLUDE}", main, "-o", DRIVER, f"-L{LIBDIR}",
               "-llbfast_b200", f"-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed: {' '.join(cmd)}\n{r.stdout}{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
