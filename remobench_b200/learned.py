"""The learned scorer's data, training and evaluation.

- collect(): stream seeded configuration-1 clouds through the plain pipeline;
  after every batch, rb_analyze logs the 16 features of every node (the
  training-data logger); when the cloud is done, each logged open node is
  paired with its final surface variation and whether it still gained points
  (the (partial, final) pairs).
- train(): Adam on those pairs with the CUDA forward/backward kernels
  (rb_mlp_train_step); nothing is trained on the CPU.
- evaluate(): at equal Refinement budgets, PSNR of the refined LOD render
  against the flat render of the same points, for the three ways of ranking the
  frontier: closure-lagged (the plain method: open nodes wait for closure),
  partial (current surface variation, no learning) and learned (open nodes by
  the network's prediction of their final surface variation).

A Refinement budget is a share of the frame's render time. Rasterizing is
bound by the samples drawn, so opening a queued node costs the samples its
children add over its own (the node's points and voxels are replaced by its
visible children's), and a budget of f admits the queue's longest prefix whose
added samples stay within f x the unrefined frame's samples.
"""
import math

import numpy as np

from . import capi, synth
from .camera import orbit_path
from .lod import Context, DeviceRing, make_frame

MIN_POINTS = 16


def _cloud(seed, num_points, batch):
    cfg = synth.config(1, seed=seed, num_points=num_points, batch_size=batch)
    pts = synth.generate(cfg)
    bmin, bmax = synth.scene_box(cfg)
    return cfg, pts, bmin, bmax


SPLIT_LIMIT = 50000  # leaf split limit: the reference's (remolod_structures.cuh:12)
SV_SCALE = 300.0    # the network's output 0 is the surface-variation correction x SV_SCALE
OFF_W3, OFF_B3 = 5248, 5376  # W3 [2][64] and b3 [2] in the parameter vector (include/rb_capi.h)


def collect(seeds, num_points=8 * 262144, batch=262144, closure_margin=2, split_limit=SPLIT_LIMIT):
    """(X, T): features of open nodes after each batch, with targets ((final -
    partial) surface variation x SV_SCALE, 1 if the node gains no further points)."""
    xs, ts = [], []
    for seed in seeds:
        cfg, pts, bmin, bmax = _cloud(seed, num_points, batch)
        ctx = Context(slot_capacity=batch, time_budget_ms=0.0, max_batches_per_build=1,
                      max_points_per_node=split_limit)
        ctx.allocate(len(pts), bmin, bmax)
        ring = DeviceRing(pts, batch, slots=ctx.cfg.ring_slots, slot_capacity=batch)
        frame = make_frame(bmin, bmax, 640, 360)
        snaps = []
        consumed = 0
        while consumed < ring.num_batches:
            ring.upload_window(consumed)
            consumed = ctx.build(ring.ring, ring.sizes, ring.uploaded, ring.num_batches).batches_consumed
            ctx.analyze(frame, min_points=MIN_POINTS, closure_margin=closure_margin)
            a = ctx.analysis()
            snaps.append((ctx.features(), a["count"].copy(), a["closed"].copy()))
        final = ctx.analysis()
        for feat, cnt, closed in snaps:
            nn = len(cnt)
            sel = (cnt >= MIN_POINTS) & (closed == 0)
            idx = np.nonzero(sel)[0]
            xs.append(feat[idx])
            # residual target: (final - partial) surface variation x SV_SCALE (feature 11 is partial x 3)
            t0 = (final["surface_variation"][:nn][idx] - feat[idx, 11] / 3.0) * SV_SCALE
            t1 = (final["count"][:nn][idx] == cnt[idx]).astype(np.float32)
            ts.append(np.stack([t0, t1], 1).astype(np.float32))
        ctx.close()
    X = np.concatenate(xs).astype(np.float32)
    T = np.concatenate(ts).astype(np.float32)
    return X, T


def train(ctx, X, T, epochs=40, batch=2048, lr=3e-3, seed=0):
    """Adam on the GPU; returns the per-epoch mean training loss."""
    import torch
    rng = np.random.default_rng(seed)
    xd = torch.from_numpy(X).cuda()
    td = torch.from_numpy(T).cuda()
    n = len(X)
    batch = max(1, min(batch, n))
    history = []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).cuda()
        xs, tsh = xd[perm].contiguous(), td[perm].contiguous()
        step_lr = lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs))
        for k in range(0, n - batch + 1, batch):
            ctx.mlp_train_step(xs[k:k + batch], tsh[k:k + batch], step_lr)
        _, loss = ctx.mlp_gradients(xd, td)
        history.append(loss)
    return history


def predict(ctx, X):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).cuda()
    y = torch.empty((len(X), 2), dtype=torch.float32, device="cuda")
    ctx.mlp_predict(xd, y)
    return y.cpu().numpy()


def mae_shrink(y, t):
    """The factor a in [0, 1] minimising sum |t - a y|: the median of t / y
    weighted by |y| (the absolute error is convex and piecewise linear in a,
    with a kink at each t / y), clipped to [0, 1]."""
    y = np.asarray(y, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    m = y != 0.0
    if not np.any(m):
        return 0.0
    r, w = t[m] / y[m], np.abs(y[m])
    order = np.argsort(r, kind="stable")
    cw = np.cumsum(w[order])
    k = int(np.searchsorted(cw, 0.5 * cw[-1]))
    return float(np.clip(r[order][min(k, len(r) - 1)], 0.0, 1.0))


def calibrate(ctx, Xval, Tval):
    """Shrinks the predicted correction toward none by the factor that gives
    the least absolute error on a validation split (mae_shrink on output 0),
    folded into the output layer's first row and bias, so the scorer never
    trusts its correction more than held-out data supports. The absolute
    error, not the squared one: the corrections are mostly near zero with a
    heavy tail, and a least-squares factor fitted to the tail adds error to
    every small one. Returns the factor."""
    y = predict(ctx, Xval)[:, 0].astype(np.float64)
    t = Tval[:, 0].astype(np.float64)
    alpha = mae_shrink(y, t)
    p = ctx.mlp_params().copy()
    p[OFF_W3:OFF_W3 + 64] *= alpha  # W3 row 0
    p[OFF_B3] *= alpha              # b3[0]
    ctx.mlp_set_params(p)
    return alpha


def psnr(a_rgba, b_rgba):
    a = a_rgba.view(np.uint8).reshape(-1, 4)[:, :3].astype(np.float64)
    b = b_rgba.view(np.uint8).reshape(-1, 4)[:, :3].astype(np.float64)
    mse = np.mean((a - b) ** 2)
    return float("inf") if mse == 0 else 10.0 * math.log10(255.0 ** 2 / mse)


def open_costs(nodes):
    """Per node, the samples opening it adds to a frame: its children's points
    and voxels minus its own (an upper bound: invisible children are culled)."""
    own = nodes["num_points"].astype(np.int64) + nodes["num_voxels"].astype(np.int64)
    kids = nodes["child"]
    add = np.zeros(len(nodes), dtype=np.int64)
    for c in range(8):
        m = kids[:, c] >= 0
        add[m] += own[kids[m, c]]
    return np.maximum(add - own, 0)


def budget_prefix(queue, costs, allowance):
    """The longest prefix of `queue` whose summed costs stay within allowance."""
    if len(queue) == 0:
        return 0
    csum = np.cumsum(costs[queue])
    return int(np.searchsorted(csum, allowance, side="right"))


def evaluate(params, seed, num_points=8 * 262144, batch=262144, stop_batch=None, closure_margin=2,
             fractions=(0.05, 0.10, 0.20, 0.40), views=3, width=960, height=540, budget_px=64.0,
             split_limit=SPLIT_LIMIT):
    """PSNR versus flat for each ranking and budget (a share of the frame's
    render time, see the module notes), averaged over `views` orbit frames, on
    the tree after `stop_batch` batches of a held-out cloud."""
    import torch
    cfg, pts, bmin, bmax = _cloud(seed, num_points, batch)
    nb = (len(pts) + batch - 1) // batch
    stop = nb // 2 if stop_batch is None else stop_batch
    ctx = Context(slot_capacity=batch, time_budget_ms=0.0, max_batches_per_build=1,
                  max_points_per_node=split_limit)
    ctx.allocate(len(pts), bmin, bmax)
    ring = DeviceRing(pts, batch, slots=ctx.cfg.ring_slots, slot_capacity=batch)
    consumed = 0
    while consumed < stop:
        ring.upload_window(consumed)
        consumed = ctx.build(ring.ring, ring.sizes, min(ring.uploaded, stop), ring.num_batches).batches_consumed
    if params is not None:
        ctx.mlp_set_params(params)
    flat_ctx = Context(pipeline=capi.RB_PIPELINE_FLAT)
    flat_ctx.allocate(len(pts), bmin, bmax)
    ingested = torch.from_numpy(pts[:consumed * batch].view(np.float32).reshape(-1, 4)).cuda()
    nodes = ctx.nodes()
    nn = len(nodes)
    costs = open_costs(nodes)
    mask = torch.zeros(nn, dtype=torch.uint8, device="cuda")
    fb = torch.empty(width * height, dtype=torch.int64, device="cuda")
    rgba = torch.empty(width * height, dtype=torch.int32, device="cuda")
    modes = {"closure_lagged": capi.RB_SCORE_CLOSED, "partial": capi.RB_SCORE_PARTIAL}
    if params is not None:
        modes["learned"] = capi.RB_SCORE_LEARNED
    out = {m: {f: [] for f in fractions} for m in modes}
    out["none"] = []
    path = orbit_path(bmin, bmax, views, seed=seed + 1000)
    frontiers, admitted = [], {m: {f: [] for f in fractions} for m in modes}
    for (yaw, pitch, rs) in path:
        frame = make_frame(bmin, bmax, width, height, yaw=yaw, pitch=pitch, radius_scale=rs, budget=budget_px)
        flat_ctx.render_flat(frame, ingested, fb, rgba)
        truth = rgba.cpu().numpy().copy()
        base = ctx.render(frame, fb, rgba)
        out["none"].append(psnr(rgba.cpu().numpy(), truth))
        # the frontier Refinement can open
        ctx.analyze(frame, min_points=MIN_POINTS, closure_margin=closure_margin, score_mode=capi.RB_SCORE_PARTIAL,
                    queue_capacity=16384)
        a = ctx.analysis()
        frontiers.append(int(np.sum(((a["flags"] & 4) != 0) & (a["count"] >= MIN_POINTS))))
        for name, mode in modes.items():
            ctx.analyze(frame, min_points=MIN_POINTS, closure_margin=closure_margin, score_mode=mode,
                        queue_capacity=16384)
            queue = ctx.queue()
            for f in fractions:
                k = budget_prefix(queue, costs, f * base.draw_samples)
                admitted[name][f].append(k)
                ctx.refine(k, mask)
                ctx.render(frame, fb, rgba, force_large=mask)
                out[name][f].append(psnr(rgba.cpu().numpy(), truth))
    frontier = float(np.mean(frontiers))
    result = {"seed": seed, "stop_batch": stop, "points": consumed * batch, "nodes": nn, "frontier": frontier,
              "psnr_none": float(np.mean(out["none"]))}
    for name in modes:
        result[name] = {f"{int(f * 100)}%": float(np.mean(out[name][f])) for f in fractions}
        result[name + "_nodes"] = {f"{int(f * 100)}%": float(np.mean(admitted[name][f])) for f in fractions}
    ctx.close()
    flat_ctx.close()
    return result


def main(argv=None):
    """Collect, train, evaluate; prints one JSON line.

    python -m remobench_b200.learned [--train-seeds 16] [--eval-seeds 4] [--points 524288]
    """
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=16)
    ap.add_argument("--eval-seeds", type=int, default=4)
    ap.add_argument("--points", type=int, default=8 * 262144)
    ap.add_argument("--batch", type=int, default=262144)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--margin", type=int, default=2)
    ap.add_argument("--split-limit", type=int, default=SPLIT_LIMIT)
    ap.add_argument("--save", default=None, help="write the trained parameters (.npy)")
    args = ap.parse_args(argv)
    t0 = time.time()
    train_seeds = list(range(100, 100 + args.train_seeds))
    eval_seeds = list(range(900, 900 + args.eval_seeds))
    X, T = collect(train_seeds, args.points, args.batch, args.margin, args.split_limit)
    Xv, Tv = collect(eval_seeds, args.points, args.batch, args.margin, args.split_limit)
    t_collect = time.time() - t0
    cfg, _, bmin, bmax = _cloud(1, args.batch, args.batch)
    ctx = Context(slot_capacity=args.batch)
    ctx.allocate(args.batch, bmin, bmax)
    ctx.mlp_init(1)
    # the last eighth of the training seeds' pairs validates the calibration
    nval = max(1, len(X) // 8)
    hist = train(ctx, X[:-nval], T[:-nval], epochs=args.epochs)
    alpha = calibrate(ctx, X[-nval:], T[-nval:])
    params = ctx.mlp_params()
    if args.save:
        np.save(args.save, params)
    pv = predict(ctx, Xv)
    # errors of the final surface variation: partial + correction, against partial alone
    sv_err_learned = float(np.mean(np.abs(pv[:, 0] - Tv[:, 0]) / SV_SCALE))
    sv_err_partial = float(np.mean(np.abs(Tv[:, 0]) / SV_SCALE))
    closure_acc = float(np.mean((pv[:, 1] > 0) == (Tv[:, 1] > 0.5)))
    evals = [evaluate(params, s, args.points, args.batch, closure_margin=args.margin, split_limit=args.split_limit)
             for s in eval_seeds]
    frontier = float(np.mean([e["frontier"] for e in evals]))
    summary = {}
    for mode in ("closure_lagged", "partial", "learned"):
        summary[mode] = {k: float(np.mean([e[mode][k] for e in evals])) for k in evals[0][mode]}
        summary[mode + "_nodes"] = {k: float(np.mean([e[mode + "_nodes"][k] for e in evals]))
                                    for k in evals[0][mode + "_nodes"]}
    print(json.dumps({"train_pairs": int(len(X)), "heldout_pairs": int(len(Xv)), "final_train_loss": hist[-1],
                      "calibration": alpha,
                      "heldout_sv_mae_learned": sv_err_learned, "heldout_sv_mae_partial": sv_err_partial,
                      "heldout_closure_accuracy": closure_acc, "psnr_no_refinement": float(np.mean([e["psnr_none"] for e in evals])),
                      "psnr": summary, "frontier_nodes": frontier, "collect_s": round(t_collect, 1),
                      "total_s": round(time.time() - t0, 1)}))


if __name__ == "__main__":
    main()
