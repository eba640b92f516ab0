"""Build libcohsearch_cuda.so in-tree for sm_100a.

``python build.py`` compiles the CUDA sources under ``csrc/`` with nvcc into
``lib/libcohsearch_cuda.so`` (the library the host packages load).  Host FP64
bookkeeping is compiled without floating-point contraction so that bin ranges
and candidate frequencies use exactly the reference's arithmetic.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["csrc/cs_api.cu", "csrc/cs_kernels.cu", "csrc/cs_synth_tc.cu", "csrc/cs_block.cu", "csrc/cs_mlp.cu"]
OUT = os.path.join(HERE, "lib", "libcohsearch_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose_ptxas=False, force=False):
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    hdrs = [os.path.join(HERE, "csrc", "cs_internal.h"), os.path.join(ROOT, "include", "cohsearch.h")]
    if not force and os.path.exists(OUT):
        newest = max(os.path.getmtime(f) for f in srcs + hdrs)
        if os.path.getmtime(OUT) >= newest:
            return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
           "-o", OUT + ".tmp", *srcs, "-lcudart"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv, force=True))
