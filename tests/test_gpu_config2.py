"""The benchmark's own workload, bit-exact against the CPU oracle: the
100M-point configuration-2 cloud (2 x 2 km, 2,000 boxes, 20,000 poles) in
1M-point batches through the reference's 50-slot ring (it wraps), 20 batches
per rb_build call with Accumulate after each -- the frame structure of
src/pipelines/RemolodPipeline.cpp:296-438 -- and three 3840 x 2160 frames of
the seeded orbit the benchmark renders.

Compared exactly, every node: node set and child structure, counters and
point/voxel counts, per-leaf point multisets with global point indices, voxel
positions with their lowest-index colours, occupancy grids, exact integer
accumulators, store offsets, and the pre-EDL packed framebuffer
(kernels/remolod/remolod_octree.cu:1062-1320, remolod_render.cu:72-198).

The oracle runs multithreaded on every host core (its threaded builder gives
the sequential builder's tree, tests/test_oracle.py).
"""
import os

import numpy as np
import pytest

from gpu_helpers import (build_gpu, compare_accums, compare_grids, compare_nodes, compare_stats, compare_voxels)
from oracle import binding as ob

pytestmark = pytest.mark.gpu

PER_CALL = 20
W, H = 3840, 2160


@pytest.fixture(scope="module")
def c2():
    from remobench_b200 import synth
    cfg = synth.config(2)
    cloud = synth.generate(cfg)
    bmin, bmax = synth.scene_box(cfg)
    bs = cfg.batch_size
    ctx, calls = build_gpu(cloud, bmin, bmax, bs, per_call=PER_CALL)
    nb = (len(cloud) + bs - 1) // bs
    tree = ob.Tree(num_threads=os.cpu_count() or 1)
    tree.reset(bmin, bmax)
    for b in range(nb):
        assert tree.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
        if (b + 1) % PER_CALL == 0 or b + 1 == nb:
            tree.accumulate(b + 1)
    tree.sweep()
    yield cfg, cloud, bmin, bmax, ctx, tree, calls
    ctx.close()
    tree.close()


def test_c2_tree_and_stats(c2):
    cfg, cloud, bmin, bmax, ctx, tree, calls = c2
    assert calls >= 5
    nodes = compare_nodes(ctx, tree)
    s = compare_stats(ctx, tree)
    assert s.num_points == len(cloud) == 100_000_000
    assert s.batchlet_index == 100 and s.mem_capacity_reached == 0 and s.overflow_flags == 0
    # the ring of 50 slots wrapped: batches 50..99 reused slots 0..49
    assert len(nodes) > 10000


def test_c2_point_multisets_with_indices(c2):
    """Every leaf's points, with their global indices, equal the oracle's as
    multisets (sorted by index on both sides)."""
    cfg, cloud, bmin, bmax, ctx, tree, _ = c2
    nodes = ctx.nodes()
    seen = 0
    for i in np.nonzero(nodes["num_points"])[0]:
        i = int(i)
        gp, gi = ctx.node_points(i)
        op, oi = tree.leaf_points(i)
        assert len(gi) == len(oi), i
        a, b = np.argsort(gi, kind="stable"), np.argsort(oi, kind="stable")
        assert np.array_equal(gi[a], oi[b]), i
        assert np.array_equal(gp.view(np.uint32).reshape(-1, 4)[a], op.view(np.uint32).reshape(-1, 4)[b]), i
        seen += len(gi)
    assert seen == len(cloud)


def test_c2_voxels_and_grids(c2):
    cfg, cloud, bmin, bmax, ctx, tree, _ = c2
    nodes = ctx.nodes()
    compare_voxels(ctx, tree, nodes)
    compare_grids(ctx, tree, nodes)


def test_c2_accumulators(c2):
    cfg, cloud, bmin, bmax, ctx, tree, _ = c2
    compare_accums(ctx, tree)
    g = ctx.accumulate(100)
    assert g.sum_leaf_counts == len(cloud) and g.inner_with_sums == 0


def test_c2_framebuffers_on_the_orbit(c2):
    """Three frames of the benchmark's seeded 300-frame orbit at 3840 x 2160,
    pre-EDL: the packed depth|colour framebuffer equals the oracle's bit for
    bit (atomicMin of the packed value is order-independent)."""
    import torch
    from remobench_b200.camera import orbit_path
    from remobench_b200.lod import make_frame
    cfg, cloud, bmin, bmax, ctx, tree, _ = c2
    path = orbit_path(bmin, bmax, 300, seed=7)
    fb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    for k in (0, 100, 200):
        yaw, pitch, rs = path[k]
        f = make_frame(bmin, bmax, W, H, yaw=yaw, pitch=pitch, radius_scale=rs)
        r = ctx.render(f, fb)
        ofr = ob.Frame()
        ofr.width, ofr.height = float(W), float(H)
        for i in range(16):
            ofr.transform[i] = f.transform[i]
            ofr.transform_frozen[i] = f.transform_frozen[i]
        for a in range(3):
            ofr.box_min[a] = f.box_min[a]
            ofr.box_max[a] = f.box_max[a]
        ofr.lod_pixel_budget = f.lod_pixel_budget
        ofr.point_size = f.point_size
        ofr.drawlist_capacity = ctx.cfg.drawlist_capacity
        ofb, orr, _ = tree.render(ofr)
        assert (r.draw_items, r.draw_samples) == (orr.draw_items, orr.draw_samples), k
        assert r.draw_samples > 1_000_000, k
        assert np.array_equal(fb.cpu().numpy().view(np.uint64), ofb), k
