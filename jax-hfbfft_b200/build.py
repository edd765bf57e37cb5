"""Build libhfb.so (sm_100a) in-tree: jax-hfbfft_b200/hfb/libhfb.so.

    python jax-hfbfft_b200/build.py [--verbose-ptxas] [-j N]

Each translation unit under csrc/ is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into build/, then linked into a
shared library with a plain C ABI (include/hfb.h).  Object files are rebuilt
only when a source or header is newer.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
OUT = os.path.join(HERE, "hfb", "libhfb.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-I", os.path.join(ROOT, "include")]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newest_dep(src):
    deps = [src] + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "hfb.h")]
    return max(os.path.getmtime(d) for d in deps)


def compile_one(src, verbose_ptxas=False):
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= _newest_dep(src) and not verbose_ptxas:
        return obj, ""
    cmd = [nvcc()] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose_ptxas=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    logs = {}
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = {ex.submit(compile_one, s, verbose_ptxas): s for s in srcs}
        objs = []
        for f in cf.as_completed(futs):
            o, log = f.result()
            objs.append(o)
            logs[futs[f]] = log
    objs.sort()
    if not os.path.exists(OUT) or max(os.path.getmtime(o) for o in objs) > os.path.getmtime(OUT):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT, logs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    out, logs = build(a.verbose_ptxas, a.j)
    if a.verbose_ptxas:
        for k, v in sorted(logs.items()):
            print(f"== {os.path.basename(k)}\n{v}")
    print(out)
    sys.exit(0)
