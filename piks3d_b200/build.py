"""Build recipe of libpiks3d_b200.so (sm_100a) and the `piks3d` command-line host.

Run `python -m piks3d_b200.build` (or call build()). Objects go to piks3d_b200/_build/,
the shared library to piks3d_b200/libpiks3d_b200.so and the CLI to piks3d_b200/bin/piks3d,
all in-tree so that they travel with the source tree. nvcc cross-compiles without a GPU.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpiks3d_b200.so")
CLI = os.path.join(HERE, "bin", "piks3d")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + CSRC,
            "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I" + CSRC,
             "-I" + os.path.join(ROOT, "include")]

CU_SOURCES = ["kernels.cu", "kernels_fp32.cu", "sweep_tile.cu", "sweep_column.cu", "preprocess.cu", "capi.cu", "batch.cu"]
CXX_SOURCES = ["host.cpp", "tiles.cpp", "output.cpp"]


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return res.stdout + res.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".inc", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def build(verbose=False, ptxas_info=False):
    """Compile every source for sm_100a and link the shared library and the CLI."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = _headers()
    objs = []
    log = ""
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            log += _run([NVCC] + CU_FLAGS + extra + ["-c", "-o", o, s])
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + hdrs):
            _run(["g++"] + CXX_FLAGS + ["-c", "-o", o, s])
        objs.append(o)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    main_src = os.path.join(CSRC, "main.cpp")
    if _stale(CLI, [main_src, LIB]):
        _run(["g++"] + CXX_FLAGS + ["-o", CLI, main_src, "-L" + HERE, "-lpiks3d_b200",
              "-Wl,-rpath,$ORIGIN/.."])
    if verbose:
        print(log)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
