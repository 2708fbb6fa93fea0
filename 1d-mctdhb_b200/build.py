"""Builds libmctdhb_b200.so (the C ABI of include/mctdhb_gpu.h) for sm_100a.

Every csrc/*.cu file is compiled by nvcc with
`-gencode arch=compute_100a,code=sm_100a` in parallel (an object is kept when
its source and headers are unchanged since its compile started), then linked
into one shared library next to this file.  Works without a GPU (cross-compile).

    python build.py [--verbose-ptxas] [--jobs N]
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmctdhb_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
         "-I" + os.path.join(REPO, "include"), "--expt-relaxed-constexpr"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def headers_mtime():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def compile_one(src, verbose_ptxas, newest_header=0.0):
    obj = os.path.join(OBJ, os.path.basename(src).replace(".cu", ".o"))
    stamp = obj + ".inputs"  # newest input mtime when the object's compile started
    newest = max(os.path.getmtime(src), newest_header)
    if not verbose_ptxas and os.path.exists(obj) and os.path.exists(stamp):
        with open(stamp) as f:
            if float(f.read() or 0) >= newest:
                return obj, ""  # up to date: built from the current source and headers
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    with open(stamp, "w") as f:
        f.write(repr(newest))
    return obj, r.stderr


def build(verbose_ptxas=False, jobs=None, quiet=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    objs = []
    newest = headers_mtime()
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, log in ex.map(lambda s: compile_one(s, verbose_ptxas, newest), srcs):
            objs.append(obj)
            if verbose_ptxas and log:
                sys.stderr.write(log)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "-Bsymbolic",
           "-Xlinker", "--no-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    build(a.verbose_ptxas, a.jobs)
