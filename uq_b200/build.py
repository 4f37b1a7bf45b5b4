"""Build the CUDA extension in-tree: uq_b200/lib/libuqlbm.so (sm_100a).

    python -m uq_b200.build

Plain nvcc (no torch extension machinery): the library exports only the C
ABI declared in include/uq_lbm.h and links the CUDA runtime statically.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(HERE, "csrc", f) for f in ("lbm_kernels.cu", "lbm_engine.cu", "lbm_noalloc.cu", "lbm_server.cu", "lbm_mat.cpp", "lbm_hdf5.cpp")]
DEPS = SRC + [os.path.join(HERE, "csrc", f) for f in ("lbm_device.cuh", "lbm_kernels.h", "lbm_host.h", "lbm_common.h", "lbm_mat.h", "lbm_hdf5.h", "tma.cuh")] + [
    os.path.join(ROOT, "include", "uq_lbm.h")]
LIB = os.path.join(HERE, "lib", "libuqlbm.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-shared",
           "-Xcompiler", "-fvisibility=hidden", "-I" + os.path.join(ROOT, "include"),
           "-o", LIB + ".tmp", *SRC, "-lz"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
