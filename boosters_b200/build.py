"""Builds libboosters_b200.so in-tree: CUDA kernels for sm_100a with nvcc,
host C++ with the system g++, statically linked CUDA runtime.

build(checked=True) builds libboosters_b200_checked.so from the same sources
with -DBST_CHECKED: device-side bounds checks that record a violation and
skip the access instead of faulting (loaded when BST_LIBRARY=checked)."""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libboosters_b200.so")
LIB_CHECKED = os.path.join(HERE, "libboosters_b200_checked.so")
BUILD_CHECKED = os.path.join(HERE, "_build_checked")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
# The system compiler has libgomp; an inherited CXX may not.
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")

# -fmad=false / -ffp-contract=off: no fused multiply-add anywhere, so f32/f64
# arithmetic rounds exactly like the reference CPU path.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
             "-Wall", "-Wno-unused-function", f"-I{CUDA}/include"]

CU_SOURCES = ["kernels.cu", "noalloc.cu", "mappers.cu"]
CPP_SOURCES = ["binning.cpp", "engine.cpp", "capi.cpp", "server.cpp", "synth.cpp", "persist.cpp", "autotune.cpp"]
HEADERS = ["kernels.h", "nvtx_range.h", "binning.h", "engine.h", "synth_gen.h", "api_util.h", "autotune.h", os.path.join("..", "..", "include", "boosters_c.h")]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose=False, checked=False):
    build_dir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    extra = ["-DBST_CHECKED"] if checked else []
    os.makedirs(build_dir, exist_ok=True)
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(build_dir, s + ".o")
        objs.append(obj)
        if _stale(obj, src):
            jobs.append([NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(build_dir, s + ".o")
        objs.append(obj)
        if _stale(obj, src):
            jobs.append([CXX] + CXX_FLAGS + extra + ["-c", src, "-o", obj])
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if jobs or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        tmp = lib + ".tmp"
        _run([CXX, "-shared", "-o", tmp] + objs +
             [f"-L{CUDA}/lib64", "-lcudart_static", "-ldl", "-lrt", "-lpthread", "-fopenmp",
              "-Wl,--no-undefined"])
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, checked="--checked" in sys.argv))
