"""Image quality of the LOD cut against the flat ground truth: the reference
names this harness but has none (README.md:183-184). Per frame, the LOD
pipeline's render and the flat pipeline's render of the same ingested points
are compared:

- psnr: peak signal-to-noise ratio of the RGB channels over the whole frame;
- coverage: of the pixels the flat render covers, the share the LOD render
  covers too (voxels stand in for the points they replace);
- depth_rel_rmse: over pixels both cover, the RMS relative depth difference.

  python -m remobench_b200.quality [--config 1 | --file cloud.simlod] [--frames 12]
                                   [--width 1920 --height 1080] [--budget 128]

prints one JSON line: the metrics per budget, as medians over the frames of a
seeded orbit.
"""
import math

import numpy as np

from . import capi

CLEAR_DEPTH_BITS = 0x7F800000  # the cleared framebuffer's depth (+inf)


def psnr(a_rgba, b_rgba):
    a = np.asarray(a_rgba).view(np.uint8).reshape(-1, 4)[:, :3].astype(np.float64)
    b = np.asarray(b_rgba).view(np.uint8).reshape(-1, 4)[:, :3].astype(np.float64)
    mse = float(np.mean((a - b) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * math.log10(255.0 ** 2 / mse)


def frame_metrics(lod_fb, flat_fb):
    """Metrics of one frame from the two packed depth|colour framebuffers (uint64)."""
    lod = np.asarray(lod_fb).view(np.uint64)
    flat = np.asarray(flat_fb).view(np.uint64)
    ld = (lod >> np.uint64(32)).astype(np.uint32)
    fd = (flat >> np.uint64(32)).astype(np.uint32)
    lcov, fcov = ld != CLEAR_DEPTH_BITS, fd != CLEAR_DEPTH_BITS
    both = lcov & fcov
    out = {"psnr": psnr((lod & np.uint64(0xFFFFFFFF)).astype(np.uint32),
                        (flat & np.uint64(0xFFFFFFFF)).astype(np.uint32)),
           "coverage": float(np.sum(both) / max(1, np.sum(fcov)))}
    if np.any(both):
        a = ld[both].view(np.float32).astype(np.float64)
        b = fd[both].view(np.float32).astype(np.float64)
        out["depth_rel_rmse"] = float(np.sqrt(np.mean(((a - b) / b) ** 2)))
    else:
        out["depth_rel_rmse"] = 0.0
    return out


def compare(ctx, flat_ctx, points_dev, frame):
    """Renders `frame` with the LOD context and the flat context over
    points_dev (the ingested points on the device); returns the metrics and
    the LOD render's sample count."""
    import torch
    n = int(frame.width) * int(frame.height)
    fb = torch.empty(n, dtype=torch.int64, device=points_dev.device)
    gt = torch.empty(n, dtype=torch.int64, device=points_dev.device)
    flat_ctx.render_flat(frame, points_dev, gt)
    r = ctx.render(frame, fb)
    m = frame_metrics(fb.cpu().numpy(), gt.cpu().numpy())
    m["samples"] = int(r.draw_samples)
    m["flat_samples"] = int(points_dev.shape[0])
    return m


def main(argv=None):
    import argparse
    import json

    import torch

    from . import synth
    from .camera import orbit_path
    from .lod import Context, DeviceRing, make_frame

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--points", type=int, default=0)
    ap.add_argument("--file", default=None, help="a .simlod cloud instead of the generator")
    ap.add_argument("--frames", type=int, default=12)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--budget", type=float, nargs="+", default=[32.0, 64.0, 128.0, 256.0])
    args = ap.parse_args(argv)
    if args.file:
        from . import simlod
        pts, bmin, bmax = simlod.load(args.file)
        batch = 1_000_000
    else:
        over = {"num_points": args.points} if args.points else {}
        cfg = synth.config(args.config, **over)
        pts = synth.generate(cfg)
        bmin, bmax = synth.scene_box(cfg)
        batch = cfg.batch_size
    ctx = Context(slot_capacity=batch, time_budget_ms=0.0)
    ctx.allocate(len(pts), bmin, bmax)
    ring = DeviceRing(pts, batch, slots=ctx.cfg.ring_slots, slot_capacity=batch)
    consumed = 0
    while consumed < ring.num_batches:
        ring.upload_window(consumed)
        consumed = ctx.build(ring.ring, ring.sizes, ring.uploaded, ring.num_batches).batches_consumed
    flat = Context(pipeline=capi.RB_PIPELINE_FLAT)
    flat.allocate(len(pts), bmin, bmax)
    dev = torch.from_numpy(np.ascontiguousarray(pts).view(np.float32).reshape(-1, 4)).cuda()
    path = orbit_path(bmin, bmax, args.frames, seed=7)
    result = {"points": int(len(pts)), "frames": args.frames, "width": args.width, "height": args.height,
              "budgets": {}}
    for budget in args.budget:
        rows = []
        for yaw, pitch, rs in path:
            f = make_frame(bmin, bmax, args.width, args.height, yaw=yaw, pitch=pitch, radius_scale=rs, budget=budget)
            rows.append(compare(ctx, flat, dev, f))
        result["budgets"][str(budget)] = {k: float(np.median([r[k] for r in rows])) for k in rows[0]}
    print(json.dumps(result))
    ctx.close()
    flat.close()


if __name__ == "__main__":
    main()
