"""Builds the native libraries of remobench_b200 in-tree (remobench_b200/lib/).

- librb_cuda.so: the CUDA kernels for sm_100a and the C ABI (include/rb_capi.h).
  Parity-critical float code (Update, Rasterize) is compiled with -fmad=false.
- librb_synth.so: the seeded synthetic lidar generator (CPU).
- librb_host.so and rb_harness: the C++ host (ILodPipeline, registry, point
  source) over the C ABI, and the headless harness.

nvcc cross-compiles without a GPU, so this runs anywhere the toolkit is.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIB = os.path.join(HERE, "lib")
BUILD = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# file -> extra flags
CUDA_UNITS = {
    "rb_update.cu": ["-fmad=false"],
    "rb_render.cu": ["-fmad=false"],
    "rb_accum.cu": [],
    "rb_capi.cu": [],
    "rb_noalloc.cu": [],
    "rb_analysis.cu": ["-fmad=false"],
    "rb_mlp.cu": [],
    "rb_refine.cu": ["-fmad=false"],
}


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    subprocess.check_call(cmd)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers(d):
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]


def build_cuda(force=False):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers(CSRC) + [os.path.join(ROOT, "include", "rb_capi.h")]
    objs = []
    for unit, extra in CUDA_UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        cmd = [nvcc] + ARCH + NVCC_FLAGS + extra + ["-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        stamp = obj + ".cmd"
        same_cmd = os.path.exists(stamp) and open(stamp).read() == " ".join(cmd)
        if force or not same_cmd or _stale(obj, [src] + hdrs):
            _run(cmd)
            with open(stamp, "w") as f:
                f.write(" ".join(cmd))
        objs.append(obj)
    out = os.path.join(LIB, "librb_cuda.so")
    if force or _stale(out, objs):
        _run([nvcc] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", out] + objs)
    return out


def build_synth(force=False):
    os.makedirs(LIB, exist_ok=True)
    src = os.path.join(CSRC, "synth.c")
    out = os.path.join(LIB, "librb_synth.so")
    if force or _stale(out, [src, os.path.join(CSRC, "synth.h")]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu11", "-o", out, src, "-lm", "-lpthread"])
    return out


def build_host(force=False):
    """The C++ host layer, if present."""
    if not os.path.isdir(HOST):
        return None
    srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp"))
    if not srcs:
        return None
    hdrs = _headers(HOST) + [os.path.join(ROOT, "include", "rb_capi.h")]
    lib_srcs = [s for s in srcs if not s.endswith("harness_main.cpp")]
    out = os.path.join(LIB, "librb_host.so")
    cuda = os.path.dirname(os.path.dirname(_nvcc()))
    common = ["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include"),
              "-I", CSRC, "-I", HOST, "-I", os.path.join(cuda, "include")]
    rpath = "-Wl,-rpath,$ORIGIN"
    # the CUDA runtime is linked statically, as nvcc links librb_cuda.so
    cudart = ["-L", os.path.join(cuda, "lib64"), "-lcudart_static", "-ldl", "-lrt", "-lpthread"]
    if force or _stale(out, lib_srcs + hdrs):
        _run(common + ["-shared", "-o", out] + lib_srcs + ["-L", LIB, "-lrb_cuda", "-lrb_synth", rpath] + cudart)
    main = os.path.join(HOST, "harness_main.cpp")
    exe = os.path.join(LIB, "rb_harness")
    if os.path.exists(main) and (force or _stale(exe, [main, out] + hdrs)):
        _run(common + ["-o", exe, main, "-L", LIB, "-lrb_host", "-lrb_cuda", "-lrb_synth", rpath] + cudart)
    return out


def build_all(force=False):
    build_synth(force)
    build_cuda(force)
    build_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built into", LIB)
