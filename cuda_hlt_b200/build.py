"""Builds the in-tree shared libraries of the package.

  libvelo_host.so  host utilities: generator, MC checker, MDF reader (g++, zlib)
  libvelo_b200.so  sm_100a kernels + C-ABI context (nvcc), linked against libvelo_host.so

The kernels are compiled with --use_fast_math, the math mode of the stage they replace
(Allen CMakeLists.txt:119), so that the float expressions kept in the reference's order
round the same way.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "--use_fast_math", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3"]


def sh(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(ext):
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(ext))


def build_host(force=False):
    lib = os.path.join(HERE, "libvelo_host.so")
    srcs = [os.path.join(CSRC, "velo_host.cpp"), os.path.join(CSRC, "velo_mdf.cpp")]
    deps = srcs + _sources(".hpp") + [os.path.join(INCLUDE, "velo_b200.h")]
    if force or _newer(lib, deps):
        sh(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-Wall", f"-I{INCLUDE}", "-o", lib] + srcs +
           ["-lpthread", "-lz"])
    return lib


def build_gpu(force=False, verbose_ptxas=False):
    lib = os.path.join(HERE, "libvelo_b200.so")
    srcs = [os.path.join(CSRC, f) for f in ("velo_chain.cu", "velo_static.cu", "velo_mlp_train.cu")]
    deps = _sources(".cu") + _sources(".cuh") + _sources(".hpp") + [os.path.join(INCLUDE, "velo_b200.h")]
    if force or _newer(lib, deps + [os.path.join(HERE, "libvelo_host.so")]):
        extra = ["-Xptxas", "-v"] if verbose_ptxas else []
        out = sh(["nvcc"] + ARCH + NVCC_FLAGS + extra + [f"-I{INCLUDE}", "-shared", "-o", lib] + srcs +
                 [f"-L{HERE}", "-lvelo_host", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"])
        if verbose_ptxas:
            print(out)
    return lib


def build(force=False):
    return [build_host(force), build_gpu(force)]


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
    if "--ptxas" in sys.argv:
        build_gpu(force=True, verbose_ptxas=True)
