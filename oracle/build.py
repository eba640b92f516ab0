"""Build the C oracle ``oracle/lib/libcs_cpu.so`` (test infrastructure).

gcc only; -ffp-contract=off so the explicit fma/fmaf calls are the only fused
operations (the reference's arithmetic), -march=x86-64-v3 for AVX2/FMA,
-fopenmp-simd for the `omp simd` lane loops of the transform (no OpenMP
runtime), pthreads for the multithreaded CPU baseline.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cs_cpu.c")
OUT = os.path.join(HERE, "lib", "libcs_cpu.so")


def build(force=False):
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-math-errno", "-fopenmp-simd", "-fPIC",
           "-shared", "-std=gnu11", "-o", OUT + ".tmp", SRC, "-lm", "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="-f" in sys.argv))
