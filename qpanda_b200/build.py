"""Build the sm_100a CUDA library in-tree: qpanda_b200/_lib/libqsb200.so.

Every .cu under qpanda_b200/csrc is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a), every host-only .cpp with g++, and
all are linked into one shared library that exports the C ABI declared in
include/qpanda_b200.h.  Beside it, qpanda_b200/_lib/libGPUEmulator.so: the
reference GPU compute unit's plug-in library (include/qpanda_b200_gpuemu.h,
qpanda_b200/host/GPUEmulatorShim.cpp) over that C ABI.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "_lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


CXX = os.environ.get("CXX_HOST", "g++")
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I" + os.path.join(ROOT, "include"),
            "-I/usr/local/cuda/include"]


def _compile(src, deps):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not _newer([src] + deps, obj):
        return obj, None
    if src.endswith(".cpp"):
        cmd = [CXX] + CXXFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "$ " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "qpanda_b200.h"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, deps), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    so = os.path.join(LIB, "libqsb200.so")
    if _newer(objs, so):
        cmd = [NVCC] + ARCH + ["-shared", "-o", so] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    shim_src = os.path.join(HERE, "host", "GPUEmulatorShim.cpp")
    shim = os.path.join(LIB, "libGPUEmulator.so")
    shim_deps = [shim_src, so, os.path.join(ROOT, "include", "qpanda_b200_gpuemu.h"),
                 os.path.join(ROOT, "include", "qpanda_b200.h")]
    if _newer(shim_deps, shim):
        cmd = [CXX] + CXXFLAGS + ["-shared", shim_src, "-o", shim, "-L" + LIB, "-lqsb200", "-ldl",
                                  "-Wl,-rpath,$ORIGIN", "-Wl,-soname,libGPUEmulator.so"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("libGPUEmulator.so failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose:
        print("built", so, "and", shim)
    return so


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
