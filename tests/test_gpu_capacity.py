"""The reference's capacity and limit paths on the B200, each against the CPU
oracle configured the same way, plus the contract checks of voxel
representatives and of kernel_accum_verify's invariants:

- ring wrap: a 3-slot ring, so batch b is read from slot b % 3
  (kernels/remolod/remolod_octree.cu:1175-1179);
- the memory check between batches (memCapacityReached, :1181-1210), also
  against the reference's own truncated run (tests/golden, recorded from its
  kernels on a B200);
- the node-pool guard that refuses splits once the pool is full (:309-321);
- the expand pass limit (:402-462), where a point's recorded leaf may be split
  after its last count and the later phases finish its descent, and point
  chunks are sized from the points that reach each leaf (the last split's
  nodes were never counted), so nothing is dropped;
- first-come voxel representatives are members of their cell, on every node;
- kernel_accum_verify's globals (remolod_accum.cu:214-233).
"""
import numpy as np
import pytest

from gpu_helpers import (build_gpu, build_oracle, compare_accums, compare_grids, compare_nodes,
                         compare_points, compare_stats, compare_voxels, gpu_view, mix64, quant28)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1_oracle(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size)
    tree.accumulate(8)
    return tree


def full_compare(ctx, tree, accums=True):
    nodes = compare_nodes(ctx, tree)
    compare_stats(ctx, tree)
    compare_points(ctx, tree, nodes)
    compare_voxels(ctx, tree, nodes)
    compare_grids(ctx, tree, nodes)
    if accums:
        compare_accums(ctx, tree)
    return nodes


def test_ring_wrap_three_slots(c1_cloud, c1_oracle):
    """Eight batches through a 3-slot ring: every build call sees at most three
    uploaded batches, the producer refills slots as they are consumed, and the
    tree equals the oracle's (which reads the cloud straight through)."""
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, calls = build_gpu(cloud, bmin, bmax, cfg.batch_size, ring_slots=3)
    assert calls >= 3
    assert ctx.stats().batchlet_index == 8
    full_compare(ctx, c1_oracle)


def test_truncation_matches_oracle_and_reference_run(c1_cloud):
    """A 230 MB store: the memory check refuses batch 5 (offset + 200 MB margin
    reaches the capacity), the build stops cleanly and reports
    memCapacityReached, and the truncated tree equals both the oracle's and the
    one the reference's own kernels built with the same store."""
    from test_ref_pin import by_key, load
    ref = load("ref_config1_ieee_store230MB.npz")
    cap = int(ref["persistent_capacity"])
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size, store_capacity=cap)
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size, persistent_capacity=cap)
    tree.accumulate(5)
    s = ctx.stats()
    assert s.batchlet_index == ref["stats_batchletIndex"] == 5
    assert s.mem_capacity_reached == 1
    assert s.persistent_capacity == cap
    assert s.persistent_offset == ref["stats_allocatedBytes_persistent"]
    assert (s.num_nodes, s.num_voxels) == (ref["stats_numNodes"], ref["stats_numVoxels"])
    full_compare(ctx, tree)
    gv, rv = by_key(gpu_view(ctx)), by_key(ref)
    assert np.array_equal(gv["keys"], rv["keys"])
    for f in ["counter", "num_points", "num_voxels", "is_leaf", "has_grid", "child_keys", "point_digest",
              "voxel_digest", "grid_digest"]:
        assert np.array_equal(gv[f], rv[f]), f
    # a later call stays stopped: nothing more is consumed
    from remobench_b200.lod import DeviceRing
    ring = DeviceRing(cloud, cfg.batch_size, slots=ctx.cfg.ring_slots, slot_capacity=cfg.batch_size)
    ring.upload_window(0)
    r = ctx.build(ring.ring, ring.sizes, ring.uploaded, ring.num_batches)
    assert r.batches_this_call == 0 and r.mem_capacity_reached == 1


@pytest.mark.parametrize("max_nodes", [201, 57])
def test_node_pool_guard_refuses_splits(c1_cloud, max_nodes):
    """A pool too small for the tree (the unbounded build makes 425 nodes):
    splits are refused once fewer than 8 ids remain, the refused leaves keep
    their points (none dropped, none duplicated), and the pool's fill and
    the node_capacity_reached flag are the oracle's."""
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size, max_nodes=max_nodes)
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size, max_nodes=max_nodes)
    tree.accumulate(8)
    full_compare(ctx, tree)
    s, o = ctx.stats(), tree.stats()
    assert s.node_capacity_reached == 1 and o.node_pool_overflow == 1
    assert max_nodes - 8 < s.num_nodes <= max_nodes
    assert s.num_points == len(cloud) and s.dropped_points == 0


@pytest.mark.parametrize("iters,graphs", [(1, 1), (2, 1), (1, 0), (3, 0)])
def test_expand_pass_limit(c1_cloud, iters, graphs):
    """max_expand_iters below what a batch needs: the loop stops with nodes
    still over the limit, points whose leaf split after their last count go on
    descending in voxel sampling and insertion, chunks cover every point that
    reaches a leaf (counters of the uncounted nodes stay 0 or lag), and every
    structure equals the oracle's with the same limit -- on the device graph
    and the host loop."""
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size, max_expand_iters=iters, use_graphs=graphs)
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size, max_expand_iters=iters)
    tree.accumulate(8)
    nodes = full_compare(ctx, tree)
    # the limit bit: some leaf ends a batch above the split threshold, and
    # some leaf holds more points than its counter says
    assert int(nodes["num_points"].max()) > 50000
    assert np.any(nodes["num_points"] > nodes["counter"])
    s = ctx.stats()
    assert s.dropped_points == 0 and s.num_points == len(cloud)


def test_first_come_representatives_are_members_of_their_cell(c1_cloud):
    """First-come mode (the reference's rule): voxel positions equal the
    oracle's, and every voxel's colour is the colour of some point of the
    ingested cloud that quantises into that voxel's own cell of that node --
    checked for every voxel of every node."""
    cfg, cloud, bmin, bmax = c1_cloud
    sub = cloud[: 3 * cfg.batch_size]
    ctx, _ = build_gpu(sub, bmin, bmax, cfg.batch_size, voxel_mode=1)
    tree = build_oracle(sub, bmin, bmax, cfg.batch_size)
    nodes = compare_nodes(ctx, tree)
    compare_voxels(ctx, tree, nodes, colours=False)
    size = float(max(np.asarray(bmax, np.float32) - np.asarray(bmin, np.float32)))
    q = np.stack([quant28(sub[a], bmin[i], size) for i, a in enumerate("xyz")], 1).astype(np.int64)
    col = sub["color"]
    levels = sorted(set(int(v) for v in nodes["level"][nodes["num_voxels"] > 0]))
    assert levels[-1] <= 14  # node and cell fit one 63-bit key below
    checked = 0
    for lv in levels:
        # each point's node at this level (a point on the box maximum wraps to
        # child 0, as the descent's bit test does) and its cell in that node
        node_xyz = (q >> (28 - lv)) & ((1 << lv) - 1)
        cell = (q >> (21 - lv)) & 127
        pkey = (((node_xyz[:, 0] << (2 * lv)) | (node_xyz[:, 1] << lv) | node_xyz[:, 2]) << 21) | \
            (cell[:, 0] + 128 * cell[:, 1] + 16384 * cell[:, 2])
        # (node, cell, colour) as one 64-bit hash; a collision could only hide a mismatch
        pkeys = np.unique(mix64(mix64(pkey) ^ col.astype(np.uint64)))
        ids = np.nonzero((nodes["level"] == lv) & (nodes["num_voxels"] > 0))[0]
        for i in ids:
            i = int(i)
            v = ctx.node_voxels(i)
            nsz = np.float64(size) / (1 << lv)
            lo = np.array([bmin[0] + nodes["X"][i] * nsz, bmin[1] + nodes["Y"][i] * nsz, bmin[2] + nodes["Z"][i] * nsz])
            pos = np.stack([v["x"], v["y"], v["z"]], 1).astype(np.float64)
            vcell = np.floor((pos - lo) / nsz * 128.0).astype(np.int64)
            assert vcell.min() >= 0 and vcell.max() < 128, i
            nk = (int(nodes["X"][i]) << (2 * lv)) | (int(nodes["Y"][i]) << lv) | int(nodes["Z"][i])
            vkey = (np.int64(nk) << 21) | (vcell[:, 0] + 128 * vcell[:, 1] + 16384 * vcell[:, 2])
            vk = mix64(mix64(vkey) ^ v["color"].astype(np.uint64))
            assert np.all(np.isin(vk, pkeys)), i
            checked += len(v)
    assert checked == int(nodes["num_voxels"].sum()) > 0


def test_accum_verify_globals(c1_cloud, c1_oracle):
    """kernel_accum_verify's invariants on the GPU: the leaves' watermarks sum
    to every stored point and no inner node holds sums."""
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size)
    g = ctx.accumulate(8)
    assert g.sum_leaf_counts == len(cloud)
    assert g.inner_with_sums == 0
    o = c1_oracle.accumulate(8)
    assert (o.sum_leaf_counts, o.inner_with_sums) == (g.sum_leaf_counts, g.inner_with_sums)
