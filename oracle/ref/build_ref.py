"""Builds the reference's own kernels and a headless launcher into oracle/_ref/.

Test infrastructure only: the outputs are the reference, run on the GPU to pin
the CPU oracle. Reads the reference sources where they lie (a read-only tree,
present only in the build container: pass its root with --reference or the
REMOBENCH_REFERENCE environment variable); writes only oracle/_ref/.

  python oracle/ref/build_ref.py --reference <reference root>

Two variants of each module (kernels/remolod/remolod_{reset,octree,accum,render}.cu):
  shipped -- the reference's NVRTC options verbatim (--use_fast_math, LTO link)
  ieee    -- the same without --use_fast_math and with --fmad=false
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref")
CUDA = "/usr/local/cuda"
MODULES = ["remolod_reset", "remolod_octree", "remolod_accum", "remolod_render"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("REMOBENCH_REFERENCE"),
                    help="root of the reference source tree (or set REMOBENCH_REFERENCE)")
    args = ap.parse_args()
    ref = args.reference
    if not ref:
        ap.error("the reference root is required: --reference or REMOBENCH_REFERENCE")
    if not os.path.isdir(os.path.join(ref, "kernels", "remolod")):
        print(f"reference sources not found under {ref}; nothing to build", file=sys.stderr)
        return 1
    os.makedirs(OUT, exist_ok=True)
    tool = os.path.join(OUT, "ref_nvrtc")
    subprocess.check_call(["g++", "-O1", "-std=c++17", f"-I{CUDA}/include", "-o", tool,
                           os.path.join(HERE, "ref_nvrtc.cpp"), f"-L{CUDA}/lib64", "-lnvrtc", "-lnvJitLink",
                           f"-Wl,-rpath,{CUDA}/lib64"])
    for m in MODULES:
        for variant in ("shipped", "ieee"):
            out = os.path.join(OUT, f"{m}.{variant}.cubin")
            subprocess.check_call([tool, os.path.join(ref, "kernels", "remolod", m + ".cu"), out,
                                   os.path.join(ref, "kernels"), os.path.join(ref, "include"), variant])
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-I{CUDA}/include",
                           f"-I{os.path.join(ref, 'kernels', 'simlod')}", f"-I{os.path.join(ref, 'include')}",
                           "-o", os.path.join(OUT, "libref_launcher.so"), os.path.join(HERE, "ref_launcher.cpp"),
                           f"-L{CUDA}/lib64/stubs", "-lcuda"])
    print("built", OUT)
    return 0


if __name__ == "__main__":
    sys.exit(main())
