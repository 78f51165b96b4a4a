"""ORACLE -- TEST INFRASTRUCTURE ONLY.

Build recipe for the checkers:

* ``oracle/_build/liboracle.so`` -- the CPU restatement ``oracle/rf_oracle.cpp``
  (g++ -O2 -ffp-contract=off, so float arithmetic is plain IEEE in source order;
  -fopenmp for the multi-threaded timing path, which is serial at one thread).
* ``oracle/_ref/libmdref_gpu.so`` -- the reference's own live kernels and host step
  functions, compiled unmodified from the reference tree for sm_100a, plus the
  harness ``oracle/ref/ref_gpu_harness.cu``.
* ``oracle/_ref/libmdref_cpu.so`` -- the reference's own CPU bond-force function
  (md_calculateforcesbpm_cpu.cpp) plus ``oracle/ref/ref_cpu_harness.cpp``.
* ``oracle/_ref/libmdref_io.so`` -- the reference's own state writers
  (md_savelammpsdata.cpp, md_savealldata.cpp, the latter with ``-include cstring``,
  which its source needs on Linux) plus ``oracle/ref/ref_io_harness.cpp``, and its
  conjugate-gradient parameter update (mp_task.h) behind ``oracle/ref/ref_fit_harness.cpp``.

The ``_ref`` builds read the reference sources where they lie: the ``ref_dir``
argument, else ``$RF_REFERENCE_DIR``, else a ``reference`` directory beside the
repository checkout. They are skipped when that tree is absent; their outputs are
git-ignored but travel with the working tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = "/usr/local/cuda/include"
# the reference checkout next to this repository's root directory
REF_BESIDE_REPO = os.path.normpath(os.path.join(HERE, "..", "..", "reference"))

# The reference translation units on the live hot path (and what they need to link).
REF_GPU_SOURCES = [
    "md_calculate_cell.cu",
    "md_cell_distribution.cu",
    "md_interaction_list_construct.cu",
    "md_interaction_list_construction.cu",
    "md_interaction_list_reconstruct.cu",
    "md_interaction_list_reconstructbpm.cu",
    "md_boundinteractions_construct.cu",
    "md_calculateforcesdem3.cu",
    "md_calculateincrementsdem.cu",
    "md_braziltest_simple2.cu",
    "md_uniaxialcompression3_simple.cu",
    "md_parallelepipedrestriction.cu",
    "md_results.cu",
]
REF_CPU_SOURCES = ["md_calculateforcesbpm_cpu.cpp"]
REF_IO_SOURCES = ["md_savelammpsdata.cpp", "md_savealldata.cpp"]


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout[-4000:], r.stderr[-4000:]))
    return r


def _newer(out, inputs):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(i) <= t for i in inputs if os.path.exists(i))


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "rf_oracle.cpp")
    hdr = os.path.join(HERE, "..", "include", "rockfit_b200.h")
    out = os.path.join(BUILD, "liboracle.so")
    if force or not _newer(out, [src, hdr, __file__]):
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-o", out, src])
    return out


def build_ref(ref_dir=None, force=False, gpu=True, cpu=True):
    ref_dir = ref_dir or os.environ.get("RF_REFERENCE_DIR") or REF_BESIDE_REPO
    if not os.path.isdir(ref_dir):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    tmp = os.path.join(REF_OUT, "obj")
    os.makedirs(tmp, exist_ok=True)
    inc = ["-I" + os.path.join(HERE, "ref"), "-I" + ref_dir]
    forced = ["-include", os.path.join(HERE, "ref", "ids32.h")]
    outs = {}
    if gpu:
        out = os.path.join(REF_OUT, "libmdref_gpu.so")
        srcs = [os.path.join(ref_dir, s) for s in REF_GPU_SOURCES]
        harness = os.path.join(HERE, "ref", "ref_gpu_harness.cu")
        if force or not _newer(out, srcs + [harness, __file__]):
            objs = []
            for s in srcs + [harness]:
                o = os.path.join(tmp, os.path.basename(s) + ".o")
                _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                      "-Xcompiler", "-fPIC", "-w"] + inc + forced + ["-c", s, "-o", o])
                objs.append(o)
            _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out] + objs +
                 ["-lcurand", "-lcudart"])
        outs["gpu"] = out
    if cpu:
        out = os.path.join(REF_OUT, "libmdref_cpu.so")
        srcs = [os.path.join(ref_dir, s) for s in REF_CPU_SOURCES]
        harness = os.path.join(HERE, "ref", "ref_cpu_harness.cpp")
        if force or not _newer(out, srcs + [harness, __file__]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-I" + CUDA_INC] + inc + forced +
                 ["-o", out] + srcs + [harness, "-lpthread"])
        outs["cpu"] = out
        out = os.path.join(REF_OUT, "libmdref_io.so")
        srcs = [os.path.join(ref_dir, s) for s in REF_IO_SOURCES]
        harness = [os.path.join(HERE, "ref", "ref_io_harness.cpp"), os.path.join(HERE, "ref", "ref_fit_harness.cpp")]
        deps = srcs + harness + [os.path.join(ref_dir, "mp_task.h"), __file__]
        if force or not _newer(out, deps):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-include", "cstring", "-I" + CUDA_INC] + inc +
                 forced + ["-o", out] + srcs + harness + ["-L/usr/local/cuda/lib64", "-lcudart"])
        outs["io"] = out
    return outs


def main():
    force = "--force" in sys.argv
    print(build_oracle(force=force))
    print(build_ref(force=force))


if __name__ == "__main__":
    main()
