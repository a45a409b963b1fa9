"""Builds the native libraries of frontistr_b200 in-tree.

  frontistr_b200/lib/libhecmw33_gpu.so     CUDA (sm_100a) solver behind the C ABI of
                                           include/hecmw33_gpu.h
  frontistr_b200/lib/libfistr_assemble.so  host C++ system generator (profile,
                                           element stiffness, boundary conditions)

Run as `python -m frontistr_b200.build`.  nvcc cross-compiles for sm_100a without
a GPU, so this works on a CPU-only machine too.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _nvcc():
    cand = os.path.join(CUDA_HOME, "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _run(cmd, cwd=None):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd, cwd=cwd)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def gpu_sources():
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".h", ".hpp")) or f.startswith("h33_")]
    srcs.append(os.path.join(ROOT, "include", "hecmw33_gpu.h"))
    return srcs


def build_gpu(force=False, verbose_ptxas=False):
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libhecmw33_gpu.so")
    cu = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
          if f.endswith(".cu") or (f.startswith("h33_") and f.endswith(".cpp"))]
    if not force and not _stale(target, gpu_sources()):
        return target
    cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-ccbin", shutil.which("g++") or "g++",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-Xcompiler", "-fopenmp", "--expt-relaxed-constexpr", "-o", target, *cu,
           "-lcudart", "-lgomp"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    _run(cmd)
    return target


def build_assemble(force=False):
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libfistr_assemble.so")
    src = os.path.join(CSRC, "assemble.cpp")
    if not force and not _stale(target, [src]):
        return target
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    _run([gxx, "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-o", target, src])
    return target


def build_all(force=False):
    return [build_assemble(force), build_gpu(force)]


if __name__ == "__main__":
    force = "--force" in sys.argv
    for p in build_all(force=force):
        print("built", p)
