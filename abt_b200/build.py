"""Builds abt_b200/libpbt_b200.so (CUDA sm_100a + host C++) in-tree.

Reference-exact translation units (k1_fp64.cu, k3_finalise.cu) are compiled
with -fmad=false and the host set-up with -ffp-contract=off, so that no
multiply-add is fused where the reference's rounding must be reproduced.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpbt_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                      "-I" + CSRC, "-I" + INCLUDE, "--expt-relaxed-constexpr",
                      "-Xptxas", "-warn-spills"]
UNITS = {
    "ctx.cu": [],
    "api.cu": [],
    "k1_fp64.cu": ["-fmad=false"],
    "k3_finalise.cu": ["-fmad=false"],
    "k2_fp32.cu": [],
    "k4_adjoint.cu": [],
}
HOST_UNITS = {"host_setup.cpp": ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
                                 "-fPIC", "-std=c++17", "-I" + CSRC, "-I" + INCLUDE,
                                 "-I" + os.path.join(CUDA_HOME, "include")],
              "beamlist.cpp": ["-O2", "-fPIC", "-std=c++17", "-I" + CSRC, "-I" + INCLUDE,
                               "-I" + os.path.join(CUDA_HOME, "include")],
              "tracer.cpp": ["-O3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
                             "-std=c++17", "-I" + CSRC, "-I" + INCLUDE,
                             "-I" + os.path.join(CUDA_HOME, "include")]}


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "pbt_diff.h"))
    return hs


def _stale(obj, src, cmd):
    """An object is rebuilt when it is missing, older than its source or a header,
    or was compiled with another command line (kept beside it in <obj>.cmd)."""
    if not os.path.exists(obj):
        return True
    try:
        with open(obj + ".cmd") as f:
            if f.read() != " ".join(cmd):
                return True
    except OSError:
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + _headers())


def _compile(unit, flags, host, verbose):
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit + ".o")
    if host:
        cmd = ["g++", "-c", src, "-o", obj] + flags
    else:
        cmd = [NVCC, "-c", src, "-o", obj] + NVCC_COMMON + flags
    if not _stale(obj, src, cmd):
        return obj
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile of %s failed:\n%s\n%s" % (unit, r.stdout, r.stderr))
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    with open(obj + ".cmd", "w") as f:
        f.write(" ".join(cmd))
    return obj


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    jobs = [(u, f, False) for u, f in UNITS.items()] + [(u, f, True) for u, f in HOST_UNITS.items()]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda j: _compile(j[0], j[1], j[2], verbose), jobs))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, "-shared", "-o", LIB] + ARCH + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print("built", LIB)
