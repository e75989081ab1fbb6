"""Times the reference's own kernels (oracle/_ref, "shipped" build) on a B200 on
the benchmark workload -- configuration 2, 100M points in 1M-point batches --
the way the reference's frame loop runs them: PointSource fills the 50-slot
ring up to its window (src/io/PointSource.cpp:223-239), kernel_construct
consumes up to 20 batches per launch under its 10 ms budget, then
kernel_accumulate (src/pipelines/RemolodPipeline.cpp:296-438). Device time of
construct + accumulate launches, CUDA events around each launch. Test
infrastructure; prints one JSON line.

  python oracle/ref/time_ref.py [--points N] [--variant shipped|ieee]
"""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def time_kernels(pts, bmin, bmax, batch_size, variant="shipped", reps=2):
    """Device time of the reference's construct + accumulate launches over the
    whole cloud `pts` (1M-point batches through its 50-slot ring). The first of
    `reps` passes warms up; the last is reported."""
    from make_ref_fixtures import Launcher, parse_stats
    lz = Launcher(variant)
    L, h = lz.L, lz.h
    vp = ctypes.c_void_p
    L.ref_construct_timed.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_float)]
    L.ref_accumulate_timed.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_float)]
    f3 = ctypes.c_float * 3
    persistent = max(48 * len(pts), 512 << 20)  # RemolodPipeline.cpp:133-135
    lz.check(L.ref_alloc(h, persistent, ctypes.byref(f3(*map(float, bmin))), ctypes.byref(f3(*map(float, bmax)))))
    bs = batch_size
    nb = (len(pts) + bs - 1) // bs
    g = (ctypes.c_uint8 * int(L.ref_sizeof(2)))()
    results = []
    try:
        for rep in range(reps):
            lz.check(L.ref_reset(h))
            uploaded, consumed = 0, 0
            construct_ms, accum_ms, launches = 0.0, 0.0, 0
            while consumed < nb:
                while uploaded < min(nb, consumed + 50):
                    chunk = np.ascontiguousarray(pts[uploaded * bs:(uploaded + 1) * bs])
                    lz.check(L.ref_upload(h, uploaded, ctypes.c_void_p(chunk.ctypes.data), len(chunk)))
                    uploaded += 1
                bi, ms, ams = ctypes.c_uint32(), ctypes.c_float(), ctypes.c_float()
                lz.check(L.ref_construct_timed(h, ctypes.byref(bi), ctypes.byref(ms)))
                lz.check(L.ref_accumulate_timed(h, ctypes.cast(g, vp), ctypes.byref(ams)))
                construct_ms += ms.value
                accum_ms += ams.value
                launches += 1
                if bi.value == consumed:
                    raise RuntimeError("construct made no progress")
                consumed = bi.value
            results.append((construct_ms, accum_ms, launches))
        sraw = (ctypes.c_uint8 * int(L.ref_sizeof(0)))()
        lz.check(L.ref_read(h, 0, ctypes.cast(sraw, vp), len(sraw), None))
        st = parse_stats(bytes(sraw))
    finally:
        lz.close()
    cms, ams, launches = results[-1]
    n = len(pts)
    return {"reference": f"kernels/remolod (NVRTC, {variant})", "points": n, "batches": nb,
            "construct_ms": round(cms, 3), "accumulate_ms": round(ams, 3), "launches": launches,
            "construct_mpts_s": round(n / cms / 1e3, 1),
            "construct_plus_accumulate_mpts_s": round(n / (cms + ams) / 1e3, 1),
            "nodes": st["numNodes"], "voxels": st["numVoxels"], "stored_points": st["numPoints"],
            "persistent_offset": st["allocatedBytes_persistent"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=100_000_000)
    ap.add_argument("--variant", default="shipped")
    args = ap.parse_args()
    from remobench_b200 import synth
    cfg = synth.config(2, num_points=args.points)
    t0 = time.time()
    pts = synth.generate(cfg)
    gen = time.time() - t0
    bmin, bmax = synth.scene_box(cfg)
    r = time_kernels(pts, bmin, bmax, cfg.batch_size, args.variant)
    r["generate_s"] = round(gen, 1)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
