"""Build the sm_100a CUDA library libslc_b200.so in-tree (nvcc, no JIT).

    python -m slchannel_b200.build          # builds if sources are newer
    python -m slchannel_b200.build --force  # always rebuilds

The library links cuFFT from the CUDA toolkit and the CUDA runtime
statically; it exports exactly the C ABI declared in include/slc_b200.h.
"""

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libslc_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "slc_b200.h")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-shared",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps.append(HEADER)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    """Compile every .cu under csrc/ into slchannel_b200/libslc_b200.so."""
    if not force and not _stale():
        return LIB
    nvcc = os.path.join(CUDA_HOME, "bin", "nvcc")
    if not os.path.exists(nvcc):
        nvcc = "nvcc"
    tmp = LIB + ".tmp"
    cmd = [nvcc, *NVCC_FLAGS]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += ["-o", tmp, *sources(), "-lcufft",
            f"-L{CUDA_HOME}/lib64", "-Xlinker", f"-rpath,{CUDA_HOME}/lib64"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libslc_b200.so:\n" + r.stdout + r.stderr)
    if ptxas_info or verbose:
        sys.stdout.write(r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
