"""In-tree build of libgalpy_cuda.so for sm_100a (B200).

``build()`` compiles galpy_b200/csrc/{galpy_cuda,orbit_kernels_more,orbit_kernels_prec,adjoint}.cu
with nvcc into galpy_b200/libgalpy_cuda.so; the library is loaded from there
by galpy_b200._lib.  Nothing is installed outside the source tree.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgalpy_cuda.so")
SOURCES = ["galpy_cuda.cu", "orbit_kernels_more.cu", "orbit_kernels_prec.cu", "adjoint.cu",
           "orbit_interp.cu"]
HEADERS = ["gpc_common.cuh", "potentials.cuh", "machines.cuh", "dop853_tableau.cuh",
           "compile_potential.h", "adjoint.cuh", "orbit_kernel.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "galpy_cuda.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the engine if any source is newer than the library (the
    translation units in parallel, then one shared-library link)."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                    "-o", LIB + ".tmp", *objs], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
