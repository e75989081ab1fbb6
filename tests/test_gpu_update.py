"""Update + Accumulate on the B200 against the CPU oracle: bit-exact node
set, per-node point multisets, occupancy bits, voxels (lowest-index rule),
statistics, and exact integer accumulators."""
import numpy as np
import pytest

from gpu_helpers import (build_gpu, build_oracle, compare_accums, compare_grids, compare_nodes,
                         compare_points, compare_stats, compare_voxels)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1_pair(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size)
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size)
    tree.accumulate(8)
    return ctx, tree


def test_tree_bit_exact(c1_pair):
    ctx, tree = c1_pair
    nodes = compare_nodes(ctx, tree)
    assert len(nodes) > 100


def test_stats_and_store_offsets(c1_pair):
    ctx, tree = c1_pair
    s = compare_stats(ctx, tree)
    assert s.num_points == 8 * 262144


def test_point_multisets(c1_pair):
    ctx, tree = c1_pair
    compare_points(ctx, tree, ctx.nodes())


def test_voxels_lowest_index(c1_pair):
    ctx, tree = c1_pair
    compare_voxels(ctx, tree, ctx.nodes())


def test_occupancy_grids(c1_pair):
    ctx, tree = c1_pair
    compare_grids(ctx, tree, ctx.nodes())


def test_accumulators_exact(c1_pair):
    ctx, tree = c1_pair
    compare_accums(ctx, tree)


def test_batch_grouping_and_host_ingest_give_same_tree(c1_cloud, c1_pair):
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, tree = c1_pair
    ref = ctx.nodes()
    # three batches per build call instead of all eight
    ctx3, calls = build_gpu(cloud, bmin, bmax, cfg.batch_size, per_call=3)
    assert calls >= 3
    assert np.array_equal(ctx3.nodes(), ref)
    compare_accums(ctx3, tree)
    # end-to-end path from host memory through the copy stream
    from remobench_b200.lod import Context
    ch = Context(slot_capacity=cfg.batch_size, time_budget_ms=0.0)
    ch.allocate(len(cloud), bmin, bmax)
    r = ch.ingest_host(cloud, cfg.batch_size)
    assert r.batches_consumed == 8
    assert np.array_equal(ch.nodes(), ref)
    compare_accums(ch, tree)


def test_first_come_voxels_are_members_of_their_cell(c1_cloud, c1_pair):
    cfg, cloud, bmin, bmax = c1_cloud
    _, tree = c1_pair
    sub = cloud[: 2 * cfg.batch_size]
    ctx, _ = build_gpu(sub, bmin, bmax, cfg.batch_size, voxel_mode=1)
    t2 = build_oracle(sub, bmin, bmax, cfg.batch_size)
    nodes = compare_nodes(ctx, t2)
    compare_voxels(ctx, t2, nodes, colours=False)
    colours = set(np.unique(sub["color"]).tolist())
    for i in np.nonzero(nodes["num_voxels"])[0][:50]:
        for v in ctx.node_voxels(int(i)):
            assert int(v["color"]) in colours


def test_host_loop_and_device_graph_agree(c1_cloud, c1_pair):
    """The host-driven expand loop (use_graphs=0, one sync per pass) and the
    device-driven batch graph (default) build the same tree and counters."""
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, tree = c1_pair
    host, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size, use_graphs=0)
    compare_nodes(host, tree)
    compare_accums(host, tree)
    a, b = host.stats(), ctx.stats()
    for f in ("num_points", "num_voxels", "num_nodes", "expand_iters", "nodes_split", "spilled_points",
              "persistent_offset", "num_allocated_chunks", "chunk_pool_size", "batchlet_index"):
        assert getattr(a, f) == getattr(b, f), f
    # both paths run the same kernels per batch and the same per-iteration
    # expand passes: on the host as launches, in the graph inside k_expand_rest
    pa = {k: v["launches"] for k, v in host.profile().items()}
    pb = {k: v["launches"] for k, v in ctx.profile().items()}
    for k in ("k_count_first", "k_deep_book", "k_deep_bin", "k_deep_split", "k_deep_move", "k_vox_sample",
              "k_insert", "k_batch_end", "expand_pass"):
        assert pa[k] == pb[k], (k, pa[k], pb[k])
    assert pa["k_split"] == pa["k_expand_cond"] == pa["expand_pass"]
    assert pb["k_expand_rest"] == pb["k_count_first"] == 8 and pb["k_split"] == 0


def test_device_time_budget_paces_but_keeps_the_tree(c1_cloud, c1_pair):
    """A 1 us device budget stops each call after its first batch; the calls
    together still build the oracle's tree."""
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, tree = c1_pair
    paced, calls = build_gpu(cloud, bmin, bmax, cfg.batch_size, time_budget_ms=0.001)
    assert calls == 8
    assert np.array_equal(paced.nodes(), ctx.nodes())
    compare_accums(paced, tree)


def test_backlog_overflow_leaves_no_stale_cells(c1_cloud):
    """A batch with more new cells than the backlog holds lists the first
    backlog_capacity of them and flags RB_OVF_BACKLOG, as the reference does at
    its limit. The cell table is empty again before the next batch: a second
    batch of the same points (which splits nodes and makes new cells of its
    own) claims every cell the first one lost, so the occupancy grids and voxel
    count end equal to the oracle's, whose 10M backlog never fills here. A cell
    left behind in the table would stay unclaimed and its bit clear."""
    cfg, cloud, bmin, bmax = c1_cloud
    first = cloud[: cfg.batch_size]
    twice = np.concatenate([first, first])
    first_cells = build_oracle(first, bmin, bmax, cfg.batch_size).stats().num_voxels
    tree = build_oracle(twice, bmin, bmax, cfg.batch_size)
    total_cells = tree.stats().num_voxels
    # the first batch overflows; the second batch's new cells (its own plus the
    # ones the first lost: total - cap) fit
    half = (total_cells + 1) // 2
    assert half < first_cells
    cap = (half + first_cells) // 2
    ctx, _ = build_gpu(twice, bmin, bmax, cfg.batch_size, backlog_capacity=cap)
    s, o = ctx.stats(), tree.stats()
    assert s.overflow_flags & 2  # RB_OVF_BACKLOG
    assert o.overflow_flags == 0
    assert (s.num_nodes, s.num_points, s.num_voxels) == (o.num_nodes, o.num_points, o.num_voxels)
    compare_grids(ctx, tree, ctx.nodes())
