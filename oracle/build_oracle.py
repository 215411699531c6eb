"""Build recipes for the test oracle (test infrastructure only).

* ``build_oracle()`` compiles this project's CPU restatement (oracle/oracle.cc) into
  ``oracle/liboracle.so``.
* ``build_ref()`` compiles the reference's own host sources -- common/graph.cc,
  common/VertexSet.cc and common/intersect.cc (AVX2, SI=0) -- where they lie in the
  reference tree, together with the project-written declaration header oracle/ref/intersect.h
  and the plan driver oracle/ref/ref_plans.cc, into ``oracle/_ref/libjref.so``.  Nothing of
  the reference is copied; when the reference tree is absent (as on a GPU box) the prebuilt
  library is used as is.

Neither library is ever loaded by the product package.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("JGPM_REFERENCE_ROOT", "/root/reference")

CXXFLAGS = ["-std=c++17", "-O3", "-fopenmp", "-fPIC", "-shared", "-march=x86-64-v3"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("oracle build failed: " + " ".join(cmd))


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def oracle_lib_path():
    return os.path.join(HERE, "liboracle.so")


def ref_lib_path():
    return os.path.join(HERE, "_ref", "libjref.so")


def build_oracle(force=False):
    out = oracle_lib_path()
    srcs = [os.path.join(HERE, "oracle.cc"), os.path.join(HERE, "rmat_oracle.h")]
    if force or _stale(out, srcs):
        _run(["g++"] + CXXFLAGS + ["-o", out, srcs[0]])
    return out


def build_ref(force=False):
    """Returns the path of libjref.so, or None when neither it nor the reference exists."""
    out = ref_lib_path()
    common = os.path.join(REF_ROOT, "common")
    if not os.path.isdir(common):
        return out if os.path.exists(out) else None
    os.makedirs(os.path.dirname(out), exist_ok=True)
    srcs = [
        os.path.join(common, "graph.cc"),
        os.path.join(common, "VertexSet.cc"),
        os.path.join(common, "intersect.cc"),
        os.path.join(HERE, "ref", "ref_plans.cc"),
    ]
    deps = srcs + [os.path.join(HERE, "ref", "intersect.h")]
    if force or _stale(out, deps):
        _run(["g++"] + CXXFLAGS + ["-mavx2", "-DSI=0", "-I", os.path.join(HERE, "ref"),
                                   "-I", os.path.join(REF_ROOT, "include"), "-o", out] + srcs)
    return out


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref(force=True))
