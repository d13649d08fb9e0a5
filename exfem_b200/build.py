"""Build ``libexfem_b200.so`` in-tree for sm_100a with nvcc.

    python exfem_b200/build.py [--verbose] [--ptxas]

Every ``csrc/*.cu`` and ``csrc/*.cpp`` file is compiled to an object under
``exfem_b200/_build/`` (in parallel, skipped when the object is newer than the
sources and headers), then linked with ``nvcc -shared`` into
``exfem_b200/libexfem_b200.so``.  ``--ptxas`` prints the register / spill /
shared-memory report of every kernel.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libexfem_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build exfem_b200")
    return exe


def _deps():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src, ptxas=False):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(p) for p in [src] + _deps())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest and not ptxas:
        return obj, ""
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
           "-I", INCLUDE, "-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd[1:1] = ["--expt-relaxed-constexpr"]
        if ptxas:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", "-O3", "-fPIC", "-std=c++17", "-I", INCLUDE, "-I", "/usr/local/cuda/include",
               "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas), srcs))
    objs = [o for o, _ in results]
    if ptxas:
        for _, log in results:
            sys.stdout.write(log)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args()
    build(verbose=True, ptxas=a.ptxas)
