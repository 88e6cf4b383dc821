"""Build libsplashtank_cuda.so in-tree for sm_100a with nvcc (python -m splashtank_b200.build).

-fmad=false keeps every float operation separately rounded, as the CPU oracle (-ffp-contract=off) does, so the
discrete results of a step (tile set, cell counts, sort order, cell types) are bit-identical.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["capi.cu", "flip_kernels.cu", "flip_extra.cu", "pbf.cu", "poisson.cu", "diff.cu", "frames.cu", "live.cu", "sdf_build.cu", "drips.cpp", "ocean.cpp"]
OUT = os.path.join(HERE, "libsplashtank_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
         "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-Xptxas", "-O3"]


def sources():
    return [os.path.join(HERE, "csrc", s) for s in SRC if os.path.exists(os.path.join(HERE, "csrc", s))]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = sources() + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(HERE, "..", "include", "splashtank_cuda.h"))
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    cmd = [NVCC] + FLAGS + sources() + ["-o", OUT + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
