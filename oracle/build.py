"""Builds the oracle libraries (test infrastructure only).

  oracle/liboracle.so            CPU restatement of the reference chain (velo_oracle.cpp); always built.
  oracle/_ref/libvelo_ref_x86.so the reference's x86 clustering, compiled from the reference tree.
  oracle/_ref/libvelo_ref_checker.so the reference's VELO track checker (checker/tracking, host
                                 code, no ROOT) with ref_checker.cpp.
  oracle/_ref/libvelo_ref_gpu.so the reference's VELO CUDA kernels, compiled from the reference tree
                                 for sm_100a with the reference's own CUDA flags (CMakeLists.txt:119:
                                 --use_fast_math --expt-relaxed-constexpr --maxrregcount=63, -O3 -DNDEBUG,
                                 separable compilation), linked with ref_harness.cu.
The _ref libraries are built only where the reference tree exists (this container); the
GPU box uses the prebuilt files, which travel with the repository snapshot.
Nothing from the reference tree is copied: sources are compiled where they lie.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference tree: VELO_REFERENCE_TREE, else a checkout named "reference" beside this
# repository. Where neither exists (the GPU box) the prebuilt _ref libraries are used as they are.
REF = os.environ.get("VELO_REFERENCE_TREE",
                     os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))
OUT = os.path.join(HERE, "_ref")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
REF_CUDA_FLAGS = ["-rdc=true", "--use_fast_math", "--expt-relaxed-constexpr", "--maxrregcount=63", "-O3", "-DNDEBUG",
                  "-lineinfo", "-Xcompiler", "-fPIC", "-std=c++17"]


def sh(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_oracle():
    src = os.path.join(HERE, "velo_oracle.cpp")
    lib = os.path.join(HERE, "liboracle.so")
    if newer(lib, [src]):
        # No FMA contraction: the restatement keeps the reference's operation order.
        sh(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", lib, src, "-lpthread"])
    return lib


def ref_includes():
    dirs = ["cuda/velo/common/include", "cuda/velo/mask_clustering/include", "cuda/velo/calculate_phi_and_sort/include",
            "cuda/velo/search_by_triplet/include", "cuda/velo/simplified_kalman_filter/include",
            "cuda/velo/consolidate_tracks/include", "cuda/event_model/velo/include", "cuda/event_model/common/include",
            "cuda/utils/sorting/include", "cuda/utils/prefix_sum/include", "cuda/utils/binary_search/include",
            "main/include", "stream/gear/include", "stream/setup/include", "cuda/event_model/UT/include",
            "cuda/event_model/SciFi/include", "cuda/UT/PrVeloUT/include", "cuda/UT/common/include",
            "cuda/SciFi/common/include", "cuda/SciFi/PrForward/include", "x86/velo/clustering/include",
            "cuda/PV/beamlinePV/include", "cuda/PV/common/include", "cuda/utils/float_operations/include",
            "cuda/global_event_cut/include"]
    return [f"-I{os.path.join(REF, d)}" for d in dirs]


def build_ref_x86():
    srcs = [os.path.join(REF, "x86/velo/clustering/src", f) for f in
            ["Clustering.cpp", "ClusteringCommon.cpp", "CudaClusteringCpuOptimized.cpp"]]
    srcs += [os.path.join(REF, "main/src/Logger.cpp"), os.path.join(REF, "main/src/Timer.cpp"),
             os.path.join(REF, "cuda/velo/common/src/ClusteringDefinitions.cu")]
    lib = os.path.join(OUT, "libvelo_ref_x86.so")
    wrapper = os.path.join(HERE, "ref_x86.cpp")
    if not newer(lib, srcs + [wrapper]):
        return lib
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-include", "array", "-DNDEBUG",
           "-I/usr/local/cuda/include"] + ref_includes() + ["-x", "c++"] + srcs + ["-x", "c++", wrapper, "-o", lib,
                                                                                   "-lpthread"]
    # ClusteringDefinitions.cu holds __device__ __host__ code; as C++ the qualifiers must vanish.
    cmd = cmd[:1] + ["-D__device__=", "-D__host__="] + cmd[1:]
    sh(cmd)
    return lib


def build_ref_checker():
    """The reference's VELO track checker (checker/tracking: TrackChecker, its categories, the
    MC associator and the MC_info reader, with main/src/Logger.cpp), host code built without
    ROOT, with ref_checker.cpp to call it."""
    srcs = [os.path.join(REF, "checker/tracking/src", f) for f in
            ("TrackChecker.cpp", "CategoriesTrackChecker.cpp", "MCAssociator.cpp", "MCEvent.cpp")]
    srcs.append(os.path.join(REF, "main/src/Logger.cpp"))
    wrapper = os.path.join(HERE, "ref_checker.cpp")
    lib = os.path.join(OUT, "libvelo_ref_checker.so")
    if newer(lib, srcs + [wrapper]):
        sh(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-I{os.path.join(REF, 'checker/tracking/include')}",
            f"-I{os.path.join(REF, 'main/include')}", "-I/usr/local/cuda/include"] + srcs + [wrapper, "-o", lib])
    return lib


def build_ref_gpu():
    kernel_dirs = ["cuda/velo/common/src", "cuda/velo/mask_clustering/src", "cuda/velo/calculate_phi_and_sort/src",
                   "cuda/velo/search_by_triplet/src", "cuda/velo/consolidate_tracks/src",
                   "cuda/velo/simplified_kalman_filter/src", "cuda/utils/prefix_sum/src", "cuda/PV/beamlinePV/src",
                   "cuda/global_event_cut/src"]
    srcs = []
    for d in kernel_dirs:
        p = os.path.join(REF, d)
        srcs += sorted(os.path.join(p, f) for f in os.listdir(p) if f.endswith(".cu"))
    harness = os.path.join(HERE, "ref_harness.cu")
    lib = os.path.join(OUT, "libvelo_ref_gpu.so")
    host_srcs = [os.path.join(REF, "x86/velo/clustering/src/ClusteringCommon.cpp"),
                 os.path.join(REF, "main/src/Logger.cpp")]
    if not newer(lib, srcs + [harness] + host_srcs):
        return lib
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    inc = ref_includes()

    def compile_one(src):
        name = os.path.basename(src)
        obj = os.path.join(objdir, name + ".o")
        extra = []
        # TrackForwarding.cu relies on VeloTools.cuh being visible at template definition
        # time (two-phase lookup of binary_search_first_candidate); nvcc 12 needs it included.
        if name == "TrackForwarding.cu":
            extra = ["-include", "VeloTools.cuh"]
        sh(["nvcc"] + ARCH + REF_CUDA_FLAGS + inc + extra + ["-c", src, "-o", obj])
        return obj

    def compile_host(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        sh(["g++", "-O3", "-std=c++17", "-fPIC", "-include", "array", "-I/usr/local/cuda/include"] + inc +
           ["-c", src, "-o", obj])
        return obj

    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        objs = list(ex.map(compile_one, srcs + [harness]))
        objs += list(ex.map(compile_host, host_srcs))
    sh(["nvcc"] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", lib] + objs + ["-lcudart"])
    shutil.rmtree(objdir, ignore_errors=True)
    return lib


def build(ref=True):
    built = [build_oracle()]
    if ref and os.path.isdir(REF):
        os.makedirs(OUT, exist_ok=True)
        built.append(build_ref_x86())
        built.append(build_ref_checker())
        built.append(build_ref_gpu())
    return built


if __name__ == "__main__":
    for b in build(ref="--no-ref" not in sys.argv):
        print(b)
