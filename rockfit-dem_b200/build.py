"""Build recipe for the engine library ``rockfit-dem_b200/lib/librfdem.so``.

CUDA sources are compiled for sm_100a only, with ``--fmad=false`` so that the
float arithmetic of the reference-mode kernels is the exact sequence of IEEE
operations the source spells out (fused multiply-adds appear only where the code
writes ``__fmaf_rn``). Host C++ is compiled with ``-ffp-contract=off`` for the same
reason. The CUDA runtime is linked statically, so the library needs only the driver.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIB_DIR, "librfdem.so")
INCLUDE = os.path.join(HERE, "..", "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU_SOURCES = ["rf_md_kernels.cu", "rf_engine.cu", "rf_pack.cu", "rf_mlp.cu"]
CXX_SOURCES = ["rf_host.cpp", "rf_io.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-ffp-contract=off", "-I" + INCLUDE]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I" + INCLUDE, "-I/usr/local/cuda/include"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout[-6000:], r.stderr[-6000:]))
    return r


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hdrs + [os.path.join(INCLUDE, "rockfit_b200.h"), __file__]


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(force=False, verbose=False):
    """Compile every source that changed and link the shared library; return its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    deps = _deps()
    objs = []
    for src in CU_SOURCES + CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, src + ".o")
        if force or _stale(obj, [path] + deps):
            if src.endswith(".cu"):
                cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
            else:
                cmd = ["g++"] + CXX_FLAGS + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
