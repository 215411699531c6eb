"""Builds libjgpm.so (the CUDA kernels and the C-ABI) in-tree for sm_100a with nvcc.

    python -m jupiter_b200.build [--force]

Objects go to jupiter_b200/_build/, the library to jupiter_b200/libjgpm.so.  Translation
units compile in parallel; a unit is rebuilt when it or any header in csrc/ or include/ is
newer than its object.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libjgpm.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                  "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src, obj, extra):
    cmd = [NVCC] + NVFLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    return src, r.returncode, r.stdout


def build(force=False, verbose=False, extra=None):
    extra = list(extra or [])
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_t = max([os.path.getmtime(h) for h in _headers()] + [0])
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            jobs.append((s, o))
    failed = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for src, rc, out in ex.map(lambda j: _compile(j[0], j[1], extra), jobs):
                if verbose or rc != 0:
                    sys.stderr.write(out)
                if rc != 0:
                    failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed: " + ", ".join(os.path.basename(f) for f in failed))
    if force or jobs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout)
            raise RuntimeError("link of libjgpm.so failed")
    build_cli(force=force or bool(jobs))
    return LIB


def build_cli(force=False):
    """The jupiter_gpm command-line front end (host C++ over the C-ABI), rpath'd to the lib."""
    src = os.path.join(PKG, "cli", "jupiter_gpm.cc")
    out = os.path.join(PKG, "jupiter_gpm")
    if not force and os.path.exists(out) and os.path.getmtime(out) > max(
            os.path.getmtime(src), os.path.getmtime(LIB)):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", out,
           "-L", PKG, "-ljgpm", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build of jupiter_gpm failed")
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
