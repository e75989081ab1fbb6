"""Refinement's deepening on the B200 against the CPU oracle's deepening of
the same queue (wiki/02_KernelPipeline.md:228-243, "local split and
redistribute"): the leaves among the Analysis queue's first entries split as
doSplitting splits a spilling node (remolod_octree.cu:303-400), their points
go one level down, voxel sampling gives the deepened nodes their voxels. The
tree, every leaf's point multiset with global indices, the voxels with their
lowest-index colours, the occupancy grids, the store offsets and the exact
accumulators equal the oracle's bit for bit -- right after the pass, and again
after two more batches build on the deepened tree."""
import numpy as np
import pytest

from gpu_helpers import compare_accums, compare_grids, compare_nodes, compare_points, compare_stats, compare_voxels
from oracle import binding as ob

pytestmark = pytest.mark.gpu

W, H = 1920, 1080


def compare_all(ctx, tree):
    nodes = compare_nodes(ctx, tree)
    compare_stats(ctx, tree)
    compare_points(ctx, tree, nodes)
    compare_voxels(ctx, tree, nodes)
    compare_grids(ctx, tree, nodes)
    compare_accums(ctx, tree)
    return nodes


@pytest.mark.parametrize("budget,min_points", [(64, 0), (40, 20000)])
def test_deepen_matches_oracle_and_later_batches_build_on_it(c1_cloud, budget, min_points):
    from remobench_b200.lod import Context, DeviceRing, make_frame
    cfg, cloud, bmin, bmax = c1_cloud
    bs = cfg.batch_size
    ctx = Context(slot_capacity=bs, time_budget_ms=0.0)
    ctx.allocate(len(cloud), bmin, bmax)
    ring = DeviceRing(cloud, bs, slots=ctx.cfg.ring_slots, slot_capacity=bs)
    ring.upload_window(0)
    assert ring.uploaded == 8
    # six batches, then the pass, then the last two
    r = ctx.build(ring.ring, ring.sizes, 6, ring.num_batches)
    assert r.batches_consumed == 6
    tree = ob.Tree()
    tree.reset(bmin, bmax)
    for b in range(6):
        assert tree.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    tree.accumulate(6)

    f = make_frame(bmin, bmax, W, H, yaw=1.2, pitch=-0.5, radius_scale=0.5)
    ctx.analyze(f, min_points=16, closure_margin=8, frontier_only=False, queue_capacity=4096)
    queue = ctx.queue()
    assert len(queue) >= budget
    before = ctx.stats()
    d = ctx.refine_deepen(budget, min_points)
    refused, taken = tree.deepen(queue[:budget], min_points)
    assert not refused and d.stopped == 0
    assert d.nodes_selected == taken and taken > 0
    assert d.nodes_split == taken and d.nodes_refused == 0
    tree.accumulate(6)
    tree.sweep()
    nodes = compare_all(ctx, tree)
    after = ctx.stats()
    assert after.num_nodes == before.num_nodes + 8 * taken
    assert (after.batchlet_index, after.num_points) == (before.batchlet_index, before.num_points)
    assert d.points_moved > 0 and d.voxels_made > 0
    g = ctx.accumulate(6)
    assert g.sum_leaf_counts == 6 * bs and g.inner_with_sums == 0
    # deepened nodes are inner now, with voxels of their own
    picked = [q for q in queue[:budget] if nodes["num_voxels"][q] > 0 and nodes["is_leaf"][q] == 0]
    assert len(picked) >= taken

    r = ctx.build(ring.ring, ring.sizes, 8, ring.num_batches)
    assert r.batches_consumed == 8
    for b in range(6, 8):
        assert tree.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    tree.accumulate(8)
    tree.sweep()
    compare_all(ctx, tree)
    ctx.close()
    tree.close()


def test_deepen_needs_analysis_and_respects_the_pool(c1_cloud):
    """The pool guard refuses splits once fewer than 8 ids remain, as in a
    batch (remolod_octree.cu:318-321), and raises the node-pool flag; the
    oracle with the same pool agrees. A pass needs a fresh Analysis queue."""
    from remobench_b200 import capi
    from remobench_b200.lod import make_frame
    from gpu_helpers import build_gpu
    cfg, cloud, bmin, bmax = c1_cloud
    sub = cloud[: 2 * cfg.batch_size]
    probe, _ = build_gpu(sub, bmin, bmax, cfg.batch_size)
    n0 = probe.stats().num_nodes
    probe.close()
    pool = n0 + 8 * 3 + 4  # room for three splits
    ctx, _ = build_gpu(sub, bmin, bmax, cfg.batch_size, max_nodes=pool)
    tree = ob.Tree(max_nodes=pool)
    tree.reset(bmin, bmax)
    for b in range(2):
        assert tree.add_batch(sub[b * cfg.batch_size:(b + 1) * cfg.batch_size]) == 0
    tree.accumulate(2)
    assert ctx.stats().num_nodes == n0
    with pytest.raises(capi.RBError):
        ctx.refine_deepen(8)
    f = make_frame(bmin, bmax, W, H, yaw=0.3, pitch=-0.6, radius_scale=0.6)
    ctx.analyze(f, min_points=16, closure_margin=8, frontier_only=False, queue_capacity=4096)
    queue = ctx.queue()
    d = ctx.refine_deepen(len(queue))
    refused, taken = tree.deepen(queue)
    assert d.nodes_selected == taken and taken > 3
    assert d.nodes_split == 3 and d.nodes_refused == taken - 3
    tree.accumulate(2)
    tree.sweep()
    compare_all(ctx, tree)
    assert ctx.stats().num_nodes == n0 + 24
    # the queue is stale after a pass
    with pytest.raises(capi.RBError):
        ctx.refine_deepen(8)
    ctx.close()
    tree.close()


def test_collapse_undoes_deepening_and_matches_oracle(c1_cloud):
    """Refinement's collapsing (wiki/02_KernelPipeline.md:228-243, "merge a
    node back up") on the B200 against the oracle: the leaves a deepening pass
    split are twigs (eight leaf children under the split limit), and
    collapsing them merges their points back, drops their voxels and returns
    their grids to the pool. Tree, points, voxels, grids, accumulators and the
    pre-EDL framebuffer equal the oracle's; two more batches then split nodes
    with the pooled grids, and the trees still agree."""
    import torch
    from test_gpu_analysis import oracle_frame
    from remobench_b200.lod import Context, DeviceRing, make_frame
    cfg, cloud, bmin, bmax = c1_cloud
    bs = cfg.batch_size
    ctx = Context(slot_capacity=bs, time_budget_ms=0.0)
    ctx.allocate(len(cloud), bmin, bmax)
    ring = DeviceRing(cloud, bs, slots=ctx.cfg.ring_slots, slot_capacity=bs)
    ring.upload_window(0)
    assert ctx.build(ring.ring, ring.sizes, 6, ring.num_batches).batches_consumed == 6
    tree = ob.Tree()
    tree.reset(bmin, bmax)
    for b in range(6):
        assert tree.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    tree.accumulate(6)
    f = make_frame(bmin, bmax, W, H, yaw=1.2, pitch=-0.5, radius_scale=0.5)
    ctx.analyze(f, min_points=16, closure_margin=8, frontier_only=False, queue_capacity=4096)
    queue = ctx.queue()
    d = ctx.refine_deepen(64)
    assert tree.deepen(queue[:64])[1] == d.nodes_selected > 0
    tree.accumulate(6)
    nodes = ctx.nodes()
    twigs = [i for i in range(1, len(nodes)) if not nodes["is_leaf"][i]
             and np.all(nodes["child"][i] >= 0) and np.all(nodes["is_leaf"][nodes["child"][i]] == 1)
             and int(nodes["num_points"][nodes["child"][i]].sum()) <= 50000]
    assert len(twigs) == d.nodes_selected
    grids_before = ctx.stats().num_grids
    r = ctx.refine_collapse(twigs + twigs[:3])
    m, moved, dropped = tree.collapse(twigs + twigs[:3])
    assert (r.nodes_collapsed, r.points_moved, r.voxels_dropped) == (m, moved, dropped)
    assert r.nodes_collapsed == len(twigs) and r.grids_returned == len(twigs)
    tree.accumulate(6)
    tree.sweep()
    compare_all(ctx, tree)
    assert ctx.stats().num_grids == grids_before - len(twigs)
    # the emptied children are reachable from no node and draw nothing
    fb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rr = ctx.render(f, fb)
    ofb, orr, _ = tree.render(oracle_frame(f))
    assert (rr.draw_items, rr.draw_samples) == (orr.draw_items, orr.draw_samples)
    assert np.array_equal(fb.cpu().numpy().view(np.uint64), ofb)

    assert ctx.build(ring.ring, ring.sizes, 8, ring.num_batches).batches_consumed == 8
    for b in range(6, 8):
        assert tree.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    tree.accumulate(8)
    tree.sweep()
    compare_all(ctx, tree)
    ctx.close()
    tree.close()


def test_deepen_is_refused_by_the_memory_check(c1_cloud):
    """A store the memory check has already closed (230 MB: the build stops
    after five of eight batches) refuses a deepening pass as it refuses a
    batch: nothing splits, `stopped` is set, and the tree still equals the
    oracle's, which refuses the same pass."""
    from test_ref_pin import load
    from gpu_helpers import build_gpu, build_oracle
    from remobench_b200.lod import make_frame
    cap = int(load("ref_config1_ieee_store230MB.npz")["persistent_capacity"])
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size, store_capacity=cap)
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size, persistent_capacity=cap)
    tree.accumulate(5)
    assert ctx.stats().mem_capacity_reached == 1
    f = make_frame(bmin, bmax, W, H, yaw=1.2, pitch=-0.5, radius_scale=0.5)
    ctx.analyze(f, min_points=16, closure_margin=8, frontier_only=False, queue_capacity=4096)
    queue = ctx.queue()
    n0 = ctx.stats().num_nodes
    d = ctx.refine_deepen(64)
    assert d.stopped == 1 and d.nodes_selected == 0 and d.nodes_split == 0
    assert tree.deepen(queue[:64]) == (True, 0)
    tree.sweep()
    assert ctx.stats().num_nodes == n0
    compare_all(ctx, tree)
    ctx.close()
    tree.close()
