"""The full streaming run (configuration 5): 1B seeded lidar points (4 x 4 km,
terrain, boxes, poles, 5% uniform outliers) streamed from pinned host memory
in 4M-point batches through rb_ingest_host, with Analysis and budgeted
Refinement every frame and the LOD cut rendered at 7680 x 4320 along three
seeded camera paths. This is the reference's frame loop (render, then build,
src/shell/App.cpp:439-444) at scale, headless.

Per frame: build the next `batches_per_frame` batches (copies from host memory
overlapped with the build on a second stream, Accumulate after them), then
Analysis, Refinement of the top `refine_fraction` of the frontier, and the
refined render with EDL. Reported: ingest rate (whole cloud / summed device
time of the ingest steps, and end to end including the host->device copies),
p50/p99 device time of the per-frame work (analysis + refine + render) and of
the whole frame, node-pool occupancy, and PSNR of the final tree's render
against the flat render of all ingested points on each camera path.

  python -m remobench_b200.streaming [--points 1000000000] [--batches-per-frame 5]
"""
import math
import time

import numpy as np

from . import capi, synth
from .camera import orbit_path
from .lod import Context, make_frame
from .quality import frame_metrics


def run(points=1_000_000_000, batch=4_000_000, batches_per_frame=5, width=7680, height=4320, max_nodes=1_000_000,
        refine_fraction=0.10, scorer_params=None, quality_frames=3, seed=1, log=None):
    import torch
    t_start = time.time()
    cfg = synth.config(5, seed=seed, num_points=points, batch_size=batch)
    bmin, bmax = synth.scene_box(cfg)
    n = cfg.num_points
    # the cloud in pinned host memory, generated in place
    host = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    view = host.numpy().view(synth.POINT_DTYPE).reshape(-1)
    synth.generate(cfg, 0, n, out=view)
    gen_s = time.time() - t_start
    if log:
        log(f"generated {n} points in {gen_s:.1f} s")

    ctx = Context(slot_capacity=batch, time_budget_ms=0.0, max_nodes=max_nodes,
                  max_batches_per_build=batches_per_frame)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.allocate(n, bmin, bmax)
    score_mode = capi.RB_SCORE_PARTIAL
    if scorer_params is not None:
        ctx.mlp_set_params(scorer_params)
        score_mode = capi.RB_SCORE_LEARNED
    mask = torch.zeros(max_nodes, dtype=torch.uint8, device="cuda")
    fb = torch.empty(width * height, dtype=torch.int64, device="cuda")
    rgba = torch.empty(width * height, dtype=torch.int32, device="cuda")

    nb = (n + batch - 1) // batch
    frames = (nb + batches_per_frame - 1) // batches_per_frame
    paths = [orbit_path(bmin, bmax, max(1, frames // 3 + 1), seed=seed + 100 + p) for p in range(3)]
    per = max(1, frames // 3 + 1)

    ingest_ms, work_ms, frame_ms, occupancy = [], [], [], []
    refined = []
    t_wall = time.time()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    for k in range(frames):
        first = k * batches_per_frame * batch
        cnt = min(batches_per_frame * batch, n - first)
        yaw, pitch, rs = paths[min(k // per, 2)][k % per]
        frame = make_frame(bmin, bmax, width, height, yaw=yaw, pitch=pitch, radius_scale=rs, edl=True)
        e0.record(stream)
        r = ctx.ingest_host(host[first:first + cnt], batch)
        e1.record(stream)
        a = ctx.analyze(frame, score_mode=score_mode, queue_capacity=16384)
        budget = int(math.ceil(refine_fraction * a.eligible))
        ctx.refine(budget, mask)
        ctx.render(frame, fb, rgba, force_large=mask)
        e2.record(stream)
        torch.cuda.synchronize()
        ingest_ms.append(e0.elapsed_time(e1))
        work_ms.append(e1.elapsed_time(e2))
        frame_ms.append(e0.elapsed_time(e2))
        refined.append(budget)
        if r.mem_capacity_reached:
            break
        occupancy.append(ctx.stats().num_nodes / max_nodes)
    wall_s = time.time() - t_wall
    stats = ctx.stats()

    # quality of the final tree against the flat render of everything ingested
    ingested = int(stats.num_points_ingested)
    flat = Context(pipeline=capi.RB_PIPELINE_FLAT)
    flat.allocate(max(ingested, 1), bmin, bmax)
    dev = host[:ingested].to("cuda", non_blocking=False)
    gt = torch.empty(width * height, dtype=torch.int64, device="cuda")
    psnr = []
    for p in range(3):
        vals = []
        for j in range(quality_frames):
            yaw, pitch, rs = paths[p][(j * per) // max(quality_frames, 1)]
            f = make_frame(bmin, bmax, width, height, yaw=yaw, pitch=pitch, radius_scale=rs)
            flat.render_flat(f, dev, gt)
            a = ctx.analyze(f, score_mode=score_mode, queue_capacity=16384)
            ctx.refine(int(math.ceil(refine_fraction * a.eligible)), mask)
            ctx.render(f, fb, force_large=mask)
            m = frame_metrics(fb.cpu().numpy(), gt.cpu().numpy())
            vals.append(m["psnr"])
        psnr.append(float(np.mean(vals)))
    del dev
    flat.close()

    total_ingest_ms = float(np.sum(ingest_ms))
    out = {
        "workload": f"config 5: {n} points (4x4 km, 8000 boxes, 80000 poles, 5% outliers) in {batch}-point batches "
                    f"from pinned host memory, {batches_per_frame} batches per frame; Analysis + Refinement "
                    f"({int(refine_fraction * 100)}% of the frontier, {'learned' if scorer_params is not None else 'partial'} "
                    f"scores) + {width}x{height} render with EDL every frame; three seeded camera paths",
        "points": n, "ingested": ingested, "frames": len(frame_ms),
        "ingest_mpts_s": round(ingested / (total_ingest_ms / 1e3) / 1e6, 1),
        "ingest_wall_mpts_s": round(ingested / wall_s / 1e6, 1),
        "frame_work_ms": {"p50": round(float(np.percentile(work_ms, 50)), 3),
                          "p99": round(float(np.percentile(work_ms, 99)), 3)},
        "frame_ms": {"p50": round(float(np.percentile(frame_ms, 50)), 3),
                     "p99": round(float(np.percentile(frame_ms, 99)), 3)},
        "refined_nodes_per_frame": {"p50": int(np.percentile(refined, 50)), "max": int(max(refined))},
        "node_pool": {"nodes": int(stats.num_nodes), "max_nodes": max_nodes,
                      "occupancy": round(stats.num_nodes / max_nodes, 4),
                      "node_capacity_reached": int(stats.node_capacity_reached)},
        "tree": {"points": int(stats.num_points), "voxels": int(stats.num_voxels), "max_depth": int(stats.max_depth),
                 "overflow_flags": int(stats.overflow_flags), "dropped": int(stats.dropped_points),
                 "mem_capacity_reached": int(stats.mem_capacity_reached)},
        "psnr_vs_flat_per_path": [round(v, 3) for v in psnr],
        "generate_s": round(gen_s, 1), "total_s": round(time.time() - t_start, 1),
    }
    ctx.close()
    return out


def main(argv=None):
    import argparse
    import json
    import sys
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=1_000_000_000)
    ap.add_argument("--batch", type=int, default=4_000_000)
    ap.add_argument("--batches-per-frame", type=int, default=5)
    ap.add_argument("--width", type=int, default=7680)
    ap.add_argument("--height", type=int, default=4320)
    ap.add_argument("--max-nodes", type=int, default=1_000_000)
    ap.add_argument("--refine", type=float, default=0.10)
    ap.add_argument("--scorer", default=None, help="trained scorer parameters (.npy): learned Refinement")
    args = ap.parse_args(argv)
    params = np.load(args.scorer) if args.scorer else None
    out = run(args.points, args.batch, args.batches_per_frame, args.width, args.height, args.max_nodes, args.refine,
              params, log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
