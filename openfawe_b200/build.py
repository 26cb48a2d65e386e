"""Build libbs_b200.so (the sm_100a CUDA library) in-tree with nvcc.

    python -m openfawe_b200.build        # or openfawe_b200.build.build()
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBRARY = os.path.join(HERE, "libbs_b200.so")
SOURCES = ["bs_context.cu", "bs_sort.cu", "bs_tree_build.cu", "bs_tree_eval.cu", "bs_direct.cu", "bs_adjoint.cu",
           "bs_tree_adjoint.cu", "bs_network.cu", "bs_operators.cu", "bs_upload.cu"]
OPENMP = {"bs_upload.cu"}  # host-threaded sources
# Sources whose FP32 pair and far-field arithmetic flushes single-precision subnormals to zero: the special-function
# results then need no subnormal handling (7% fewer instructions in the interaction-list kernel); FP64 is unaffected,
# and an FP32 value below 1.2e-38 m/s is no part of a velocity here (out-of-range pairs are evaluated in FP64).
FTZ = {"bs_tree_eval.cu", "bs_direct.cu", "bs_tree_adjoint.cu"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA library cannot be built")
    return path


def build(verbose=False, extra=()):
    """Compile every source to an object under csrc/_build and link the shared library; returns its path."""
    out_dir = os.path.join(CSRC, "_build")
    os.makedirs(out_dir, exist_ok=True)
    objects = []
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "bs_b200.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)
    for source in SOURCES:
        src = os.path.join(CSRC, source)
        obj = os.path.join(out_dir, source.replace(".cu", ".o"))
        objects.append(obj)
        if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= newest_header and not extra):
            continue
        omp = ["-Xcompiler", "-fopenmp"] if source in OPENMP else []
        ftz = ["-ftz=true"] if source in FTZ else []
        cmd = [nvcc(), *ARCH, *FLAGS, *omp, *ftz, *extra, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if (not os.path.exists(LIBRARY) or extra
            or any(os.path.getmtime(o) > os.path.getmtime(LIBRARY) for o in objects)):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIBRARY, *objects, "-Xcompiler", "-fopenmp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIBRARY


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
