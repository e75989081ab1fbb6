"""Covariance precision by octree depth on a UTM-offset, millimetre-quantised
cloud: this path's exact integer sums against three float schemes.

The cloud is configuration 3 of the generator: world coordinates at
(500000, 4000000) m, snapped to 1 mm, with 0.5 mm range noise so surfaces are
close to planar and the smallest eigenvalue is tiny. The tree is built on the
GPU from float32 coordinates relative to the box minimum (as the reference's
readers store them), Analysis rolls the exact integer sums up and takes the
eigenvalues. For the same subtree of every node, four estimates are compared
with a float64 truth computed from the float64 world coordinates centred on
the node's own minimum corner:

- int64:        this path (rb_analyze; exact 28-bit sums, FP32/FP64 eigen solve)
- fp32 naive:   float32 sums of float32 world coordinates (Σx, Σxxᵀ, then
                C = Σxxᵀ/n − x̄x̄ᵀ)
- fp32 centred: float32 sums of float32 node-local coordinates
- fp64 ref:     float64 sums of node-normalised coordinates in [0, 1] taken
                from the stored float32 points, the reference's Accumulate
                scheme (kernels/remolod/remolod_accum.cu:115-153)

All sums are accumulated on the GPU (torch index_add_). Reported per depth:
the median and 95th-percentile relative error of the smallest eigenvalue and
of the surface variation, and the share of nodes whose smallest eigenvalue
comes out non-positive or more than 100% off.

python -m remobench_b200.precision [--points 20000000] [--min-points 64]
"""
import argparse
import json
import time

import numpy as np

from . import synth
from .lod import Context, make_frame


def _ancestors(nodes):
    """(nn, 21) table: ancestor id at each level (self at its own level, -1 below)."""
    nn = len(nodes)
    parent = np.full(nn, -1, dtype=np.int64)
    ch = nodes["child"]
    for k in range(8):
        c = ch[:, k]
        ok = c >= 0
        parent[c[ok]] = np.nonzero(ok)[0]
    level = nodes["level"].astype(np.int64)
    anc = np.full((nn, 21), -1, dtype=np.int64)
    cur = np.arange(nn)
    curlev = level.copy()
    while True:
        ok = cur >= 0
        if not ok.any():
            break
        anc[np.nonzero(ok)[0], curlev[ok]] = cur[ok]
        nxt = np.where(ok, parent[np.maximum(cur, 0)], -1)
        curlev = curlev - 1
        cur = np.where(curlev >= 0, nxt, -1)
    return anc


def _cov_from_sums(n, s1, s2):
    """Covariance (K, 3, 3) from counts, first sums (K, 3) and second sums (K, 6: xx xy xz yy yz zz)."""
    import torch
    m = s1 / n[:, None]
    c = torch.empty((len(n), 3, 3), dtype=torch.float64, device=s1.device)
    idx = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    for k, (a, b) in enumerate(idx):
        v = s2[:, k].double() / n - m[:, a].double() * m[:, b].double()
        c[:, a, b] = v
        c[:, b, a] = v
    return c


def _sums(vals, seg, nseg, dtype):
    import torch
    v = vals.to(dtype)
    s1 = torch.zeros((nseg, 3), dtype=dtype, device=v.device)
    s1.index_add_(0, seg, v)
    prods = torch.stack([v[:, 0] * v[:, 0], v[:, 0] * v[:, 1], v[:, 0] * v[:, 2],
                         v[:, 1] * v[:, 1], v[:, 1] * v[:, 2], v[:, 2] * v[:, 2]], 1)
    s2 = torch.zeros((nseg, 6), dtype=dtype, device=v.device)
    s2.index_add_(0, seg, prods)
    return s1, s2


def run(num_points=20_000_000, min_points=64, seed=1, batch=1_000_000):
    import torch
    t0 = time.time()
    cfg = synth.config(3, num_points=num_points, range_noise=0.0005, seed=seed)
    pts = synth.generate(cfg)                      # float32, relative to the box minimum
    xyz64, _ = synth.generate_f64(cfg)             # float64 world coordinates
    bmin, bmax = synth.scene_box(cfg)
    info_min = synth.scene_box_f64(cfg)[0]               # world box minimum, float64
    t_gen = time.time() - t0

    ctx = Context(slot_capacity=batch, time_budget_ms=0.0)
    ctx.allocate(len(pts), bmin, bmax)
    ctx.ingest_host(pts, batch)
    frame = make_frame(bmin, bmax, 1920, 1080)
    ctx.analyze(frame, min_points=min_points, frontier_only=False)
    an = ctx.analysis()
    nodes = ctx.nodes()
    nn = len(nodes)
    size = float(max(bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2]))

    # every point's leaf, from the leaves' global indices
    leaf_of = np.full(len(pts), -1, dtype=np.int64)
    for i in np.nonzero(nodes["num_points"])[0]:
        _, idx = ctx.node_points(int(i))
        leaf_of[idx] = i
    assert (leaf_of >= 0).all(), "a point is in no leaf"
    anc = _ancestors(nodes)

    dev = torch.device("cuda")
    w64 = torch.from_numpy(xyz64).to(dev)                          # world, float64
    rel32 = torch.from_numpy(pts.view(np.float32).reshape(-1, 4)[:, :3].copy()).to(dev)
    w32 = w64.float()                                               # world, float32
    level = nodes["level"].astype(np.int64)
    nsize = size / np.exp2(level)                                   # node edge in metres
    nmin_rel = np.stack([nodes["X"], nodes["Y"], nodes["Z"]], 1) * nsize[:, None]
    nmin_rel = np.asarray(nmin_rel, dtype=np.float64) + np.asarray(bmin, dtype=np.float64)
    nmin_world = nmin_rel + info_min                                # node minimum corner, world

    per_depth = {}
    for d in range(int(level.max()) + 1):
        a = anc[leaf_of, d]
        ok = a >= 0
        seg_np = a[ok]
        sel = torch.from_numpy(np.nonzero(ok)[0]).to(dev)
        uniq, inv = np.unique(seg_np, return_inverse=True)
        seg = torch.from_numpy(inv).to(dev)
        k = len(uniq)
        cnt = torch.zeros(k, dtype=torch.float64, device=dev)
        cnt.index_add_(0, seg, torch.ones(len(seg), dtype=torch.float64, device=dev))
        origin = torch.from_numpy(nmin_world[uniq]).to(dev)
        sz = torch.from_numpy(nsize[uniq]).to(dev)
        # truth: float64, centred on the node's corner
        loc64 = w64[sel] - origin[seg]
        t1, t2 = _sums(loc64, seg, k, torch.float64)
        c_true = _cov_from_sums(cnt, t1, t2)
        # fp32 naive: float32 world coordinates
        n1, n2 = _sums(w32[sel], seg, k, torch.float32)
        c_naive = _cov_from_sums(cnt, n1.double(), n2.double())
        # fp32 centred: float32 node-local coordinates
        c1_, c2_ = _sums(loc64.float(), seg, k, torch.float32)
        c_cent = _cov_from_sums(cnt, c1_.double(), c2_.double())
        # fp64 reference scheme: node-normalised [0, 1] from the stored float32 points
        orel = torch.from_numpy(nmin_rel[uniq] - np.asarray(bmin, dtype=np.float64)).to(dev)
        unit = ((rel32[sel].double() - torch.from_numpy(np.asarray(bmin, np.float64)).to(dev)) - orel[seg]) / sz[seg, None]
        unit = unit.clamp(0.0, 1.0)
        r1, r2 = _sums(unit, seg, k, torch.float64)
        c_ref = _cov_from_sums(cnt, r1, r2) * (sz ** 2)[:, None, None]

        keep = (cnt >= min_points)
        ev_true = torch.linalg.eigvalsh(c_true)            # ascending
        lmin_true = ev_true[:, 0]
        sv_true = lmin_true / ev_true.sum(1)
        keep = keep & (lmin_true > 0)
        res = {"nodes": int(keep.sum())}
        if res["nodes"] == 0:
            continue

        def errs(lmin, sv):
            e_l = ((lmin - lmin_true).abs() / lmin_true)[keep].cpu().numpy()
            e_s = ((sv - sv_true).abs() / sv_true)[keep].cpu().numpy()
            bad = ((lmin <= 0) | ((lmin - lmin_true).abs() > lmin_true))[keep].float().mean().item()
            return {"lmin_rel_median": float(np.median(e_l)), "lmin_rel_p95": float(np.percentile(e_l, 95)),
                    "sv_rel_median": float(np.median(e_s)), "sv_rel_p95": float(np.percentile(e_s, 95)),
                    "failed_share": bad}

        for name, c in (("fp32_naive", c_naive), ("fp32_centred", c_cent), ("fp64_ref", c_ref)):
            ev = torch.linalg.eigvalsh(c)
            res[name] = errs(ev[:, 0], ev[:, 0] / ev.sum(1))
        # this path: eigenvalues in (node size)^2, descending
        ids = torch.from_numpy(uniq).long()
        eig = torch.from_numpy(an["eig"][ids.numpy()].astype(np.float64)).to(dev) * (sz ** 2)[:, None]
        sv_ours = torch.from_numpy(an["surface_variation"][ids.numpy()].astype(np.float64)).to(dev)
        res["int64"] = errs(eig[:, 2], sv_ours)
        per_depth[d] = res
    out = {"points": int(len(pts)), "nodes": int(nn), "octree_size_m": size,
           "world_min": [float(v) for v in info_min], "generate_s": round(t_gen, 1),
           "total_s": round(time.time() - t0, 1), "per_depth": per_depth}
    ctx.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=20_000_000)
    ap.add_argument("--min-points", type=int, default=64)
    args = ap.parse_args(argv)
    print(json.dumps(run(args.points, args.min_points)))


if __name__ == "__main__":
    main()
