"""Builds libsmoq_cuda.so in-tree for sm_100a (and, for tests, the CPU oracle).

    python smoq.jl_b200/build.py            # CUDA library + oracle
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib", "libsmoq_cuda.so")
SOURCES = ["capi.cu", "k_kernels.cu", "k_stage.cu", "planner.cpp", "mcwf.cu", "vqe.cu", "noalloc.cu", "measure.cu", "dm.cu", "qrc.cu", "circuit.cu", "noisy_grad.cu", "jit.cpp"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC"]
OBJDIR = os.path.join(PKG, "_build")


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(force=False, verbose=False, lib=LIB, defines=()):
    """Compile every source to an object (in parallel), link the shared library.
    `defines` (e.g. ["SMOQ_STAGE_MINB_C64=2"]) are passed as -D to every source."""
    srcs = _sources()
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "smoq_cuda.h"))
    if not force and not defines and not _stale(lib, deps):
        return lib
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    dflags = ["-D" + d for d in defines]
    tag = "_".join(d.replace("=", "") for d in defines)

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.basename(src) + (("." + tag) if tag else "") + ".o")
        cmd = [nvcc] + NVCC_FLAGS + dflags + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", obj, src]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, srcs))
    for obj, r in results:
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        if verbose:
            sys.stderr.write(r.stderr)
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib] +
                       [o for o, _ in results], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    return lib


def build_oracle(force=False):
    odir = os.path.join(ROOT, "oracle")
    target = os.path.join(odir, "libsmoq_oracle.so")
    deps = [os.path.join(odir, f) for f in ("smoq_oracle.c", "smoq_oracle.h", "Makefile")]
    if not force and not _stale(target, deps):
        return target
    r = subprocess.run(["make", "-C", odir, "-B"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return target


if __name__ == "__main__":
    print(build_cuda(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_oracle(force="--force" in sys.argv))
