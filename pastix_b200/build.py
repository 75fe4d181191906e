"""Build the CUDA library libpastix_gpu.so in-tree for sm_100a (B200).

    python -m pastix_b200.build

nvcc cross-compiles without a GPU; the shared object lands in
pastix_b200/lib/ next to this file, which is where pastix_b200.gpu loads it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpastix_gpu.so")
PEAKLIB = os.path.join(LIBDIR, "libpgpu_peak.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["pastix_gpu.cu", "pgpu_mlp.cu", "pgpu_analysis.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "pastix_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIBDIR, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", CSRC,
                                       "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    # bench-only helper: FMA peak microbenchmark
    subprocess.check_call([NVCC] + ARCH + FLAGS + ["-shared", "-o", PEAKLIB, os.path.join(CSRC, "peak.cu")])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
