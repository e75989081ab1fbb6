"""The CPU oracle against hand-derived known answers and the reference's own
invariants (the reference ships no tests or fixtures for this path; its
structural pins are on lidar files that are not distributed)."""
import numpy as np
import pytest

from oracle import binding as ob

PT = ob.POINT_DTYPE


def pts(rows):
    a = np.zeros(len(rows), dtype=PT)
    for i, (x, y, z, c) in enumerate(rows):
        a[i] = (x, y, z, c)
    return a


def unit_tree(**cfg):
    t = ob.Tree(**cfg)
    t.reset((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    return t


def test_child_index_bit_order():
    # remolod_octree.cu:184-192: child = (x << 2) | (y << 1) | z of bit (19 - level).
    # (0.75, 0.25, 0.5) in a unit cube: X20 = 786432 (bit19=1), Y20 = 262144 (0), Z20 = 524288 (1) -> child 5.
    t = unit_tree(max_points_per_node=4)
    cloud = pts([(0.75, 0.25, 0.5, 1), (0.25, 0.25, 0.25, 2), (0.25, 0.75, 0.25, 3),
                 (0.75, 0.75, 0.75, 4), (0.25, 0.25, 0.75, 5)])
    assert t.add_batch(cloud) == 0
    t.sweep()
    root = t.node(0)
    assert not root.is_leaf
    kids = list(root.child)
    assert kids == list(range(1, 9))  # the first split takes ids 1..8
    c5 = t.node(kids[5])
    assert (c5.level, c5.X, c5.Y, c5.Z) == (1, 1, 0, 1)
    assert c5.num_points == 1 and c5.counter == 1
    p, idx = t.leaf_points(kids[5])
    assert list(idx) == [0]
    assert [t.node(k).num_points for k in kids] == [1, 1, 1, 0, 0, 1, 0, 1]


def test_root_voxel_cell_and_centre():
    # sampleVoxel (remolod_octree.cu:103-133) at the root, level 0: cell = pFull >> 21.
    # pFull = u32(2^28 * 0.75) = 201326592 -> 96; 0.25 -> 32; 0.5 -> 64.
    # centre x = 0 + 1 * (96 + 0.5) / 128 = 0.75390625.
    t = unit_tree(max_points_per_node=4)
    cloud = pts([(0.75, 0.25, 0.5, 0xAABBCCDD)] * 5)
    t.add_batch(cloud)
    g = t.node_grid(0)
    vi = 96 + 32 * 128 + 64 * 16384
    assert g[vi // 32] == (1 << (vi % 32))
    assert int(np.count_nonzero(g)) == 1
    v = t.node_voxels(0)
    assert len(v) == 1
    assert v[0]["x"] == np.float32(0.75390625)
    assert v[0]["y"] == np.float32((32 + 0.5) / 128)
    assert v[0]["z"] == np.float32((64 + 0.5) / 128)
    assert v[0]["color"] == 0xAABBCCDD


def test_box_max_wraps_to_cell_zero():
    # A point exactly on boxMax quantises to 2^20: the descent's per-level & 1
    # wraps it to the low child (wiki/04_FixedDepthFindings.md:291-296), and
    # its 2^28 cell index wraps to 0 at the root (% 128).
    t = unit_tree(max_points_per_node=2)
    cloud = pts([(1.0, 1.0, 1.0, 7), (1.0, 1.0, 1.0, 8), (1.0, 1.0, 1.0, 9)])
    t.add_batch(cloud)
    root = t.node(0)
    assert not root.is_leaf
    # child 0 (x=y=z=0) holds them, and so on down to MAX_DEPTH: every level wraps
    c0 = t.node(root.child[0])
    assert c0.counter == 3
    g = t.node_grid(0)
    assert g[0] & 1


def test_lowest_index_representative():
    t = unit_tree(max_points_per_node=8)
    # 9 points in one root cell, different colours; the first (lowest index) wins
    cloud = pts([(0.1, 0.1, 0.1 + 1e-6 * i, 100 + i) for i in range(9)])
    t.add_batch(cloud)
    v = t.node_voxels(0)
    assert len(v) == 1 and v[0]["color"] == 100


def test_spilled_points_keep_index_and_win_later_cells():
    # batch 0 fills a leaf to the limit; batch 1 pushes it over: the stored points
    # spill and re-insert into children with their original indices.
    t = unit_tree(max_points_per_node=4)
    b0 = pts([(0.6 + 0.01 * i, 0.6, 0.6, 10 + i) for i in range(4)])
    b1 = pts([(0.6 + 0.01 * i, 0.6, 0.6, 20 + i) for i in range(2)])
    t.add_batch(b0)
    assert t.node(0).is_leaf
    t.add_batch(b1)
    t.sweep()
    s = t.stats()
    assert s.num_points == 6 and s.spilled_points == 4
    seen = {}
    for i in range(t.num_nodes()):
        p, idx = t.leaf_points(i)
        for q, k in zip(p, idx):
            seen[int(k)] = int(q["color"])
    assert seen == {0: 10, 1: 11, 2: 12, 3: 13, 4: 20, 5: 21}


def test_node_pool_refusal_keeps_points():
    t = unit_tree(max_points_per_node=2, max_nodes=9)
    cloud = pts([(0.1 * (i % 9) + 0.05, 0.3, 0.3, i) for i in range(30)])
    t.add_batch(cloud)
    t.sweep()
    s = t.stats()
    assert s.node_pool_overflow == 1
    assert s.num_nodes == 9
    assert s.num_points == 30  # nothing dropped, nothing duplicated
    assert s.dropped_points == 0


def test_memory_check_truncates_between_batches():
    # AllocatorGlobal offsets (utils.h.cu:195): root grid 262160 B after the 16-byte header;
    # a capacity below offset + margin refuses the batch (remolod_octree.cu:1197-1210).
    t = ob.Tree(persistent_capacity=16 + 262160 + 1000, safety_margin=1000)
    t.reset((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    assert t.stats().persistent_offset == 16 + 262160
    cloud = pts([(0.5, 0.5, 0.5, 1)])
    assert t.add_batch(cloud) == 1
    assert t.stats().mem_capacity_reached == 1
    assert t.stats().batchlet_index == 0


def test_config1_invariants(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    t = ob.Tree()
    t.reset(bmin, bmax)
    bs = cfg.batch_size
    for b in range(8):
        assert t.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    t.sweep()
    s = t.stats()
    n = len(cloud)
    # diagnostics() invariants (src/pipelines/RemolodPipeline.cpp:603-726)
    assert s.num_points == n
    assert s.counter_underflows == 0
    assert s.dropped_points == 0 and s.overflow_flags == 0
    assert s.num_inner + s.num_leaves == s.num_nodes
    g = t.accumulate(8)
    assert g.sum_leaf_counts == n
    assert g.inner_with_sums == 0
    # every input point is stored exactly once, with its global index
    seen = np.zeros(n, dtype=np.int32)
    nodes = t.node_table()
    for i in np.nonzero(nodes["is_leaf"])[0]:
        p, idx = t.leaf_points(int(i))
        seen[idx] += 1
        assert np.array_equal(p.view(np.uint32).reshape(-1, 4), cloud[idx].view(np.uint32).reshape(-1, 4))
    assert np.all(seen == 1)
    # leaves stay within the split limit unless they sit at MAX_DEPTH
    assert np.all(nodes["num_points"][nodes["is_leaf"] == 1] <= 50000)


def test_build_ring_equals_add_batch(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    sub = cloud[: 4 * cfg.batch_size]
    bs = cfg.batch_size
    a = ob.Tree()
    a.reset(bmin, bmax)
    for b in range(4):
        a.add_batch(sub[b * bs:(b + 1) * bs])
    a.sweep()
    # the same batches through kernel_construct's ring loop, two at a time
    ring = np.zeros(50 * bs, dtype=ob.POINT_DTYPE)
    sizes = np.zeros(50, dtype=np.uint32)
    for b in range(4):
        ring[b * bs:(b + 1) * bs] = sub[b * bs:(b + 1) * bs]
        sizes[b] = bs
    t = ob.Tree(slot_capacity=bs, max_batches_per_build=2)
    t.reset(bmin, bmax)
    assert t.build(ring, sizes, 4) == 2
    assert t.build(ring, sizes, 4) == 2
    assert np.array_equal(a.node_table(), t.node_table())


def test_accumulate_watermark_is_incremental(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    bs = cfg.batch_size
    once = ob.Tree()
    once.reset(bmin, bmax)
    twice = ob.Tree()
    twice.reset(bmin, bmax)
    for b in range(3):
        once.add_batch(cloud[b * bs:(b + 1) * bs])
        twice.add_batch(cloud[b * bs:(b + 1) * bs])
        twice.accumulate(b)
    once.accumulate(2)
    for i in range(once.num_nodes()):
        a, b = once.accum_i(i), twice.accum_i(i)
        assert bytes(a)[:-12] == bytes(b)[:-12]  # all sums and the count; not last_touched_batch


def test_jacobi_known_eigenvalues():
    e, v = ob.sym3_eig([2.0, 0.0, 0.0, 3.0, 0.0, 1.0])
    assert np.allclose(e, [3.0, 2.0, 1.0])
    assert np.allclose(np.abs(v), [0.0, 0.0, 1.0])
    a = np.array([[4.0, 1.0, 0.5], [1.0, 3.0, 0.2], [0.5, 0.2, 1.0]])
    e, _ = ob.sym3_eig([a[0, 0], a[0, 1], a[0, 2], a[1, 1], a[1, 2], a[2, 2]])
    assert np.allclose(e, np.sort(np.linalg.eigvalsh(a))[::-1], rtol=1e-12)


def test_threaded_builder_matches_sequential(c1_cloud):
    """The multithreaded CPU builder (the timed CPU baseline) builds the same
    tree, points and voxels, in the same order, as the sequential one."""
    cfg, cloud, bmin, bmax = c1_cloud
    sub = cloud[: 4 * cfg.batch_size]
    trees = []
    for threads in (1, 4):
        t = ob.Tree(num_threads=threads)
        t.reset(bmin, bmax)
        for b in range(4):
            assert t.add_batch(sub[b * cfg.batch_size:(b + 1) * cfg.batch_size]) == 0
        t.sweep()
        trees.append(t)
    a, b = trees
    assert np.array_equal(a.node_table(), b.node_table())
    for i in range(a.num_nodes()):
        pa, ia = a.leaf_points(i)
        pb, ib = b.leaf_points(i)
        assert np.array_equal(ia, ib) and np.array_equal(pa.view(np.uint32), pb.view(np.uint32))
        assert np.array_equal(a.node_voxels(i).view(np.uint32), b.node_voxels(i).view(np.uint32))


def test_colour_filtering_known_answer():
    # five points in one root cell (128^3 grid of a unit cube) split the root
    # (limit 4); the root keeps one voxel for the cell, coloured by the lowest
    # index; filtering makes it the mean of the five points, rounded half up
    t = unit_tree(max_points_per_node=4)
    cols = [(10, 20, 30), (20, 30, 40), (30, 40, 51), (40, 50, 60), (51, 60, 70)]
    cloud = pts([(0.3 + 0.0005 * i, 0.6, 0.6, r | (g << 8) | (b << 16) | (200 << 24))
                 for i, (r, g, b) in enumerate(cols)])
    t.add_batch(cloud)
    t.sweep()
    assert not t.node(0).is_leaf
    v = t.node_voxels(0)
    assert len(v) == 1 and int(v[0]["color"]) == int(cloud[0]["color"])
    m, nv = t.refine_colors([0])
    assert (m, nv) == (1, 1)
    c = int(t.node_voxels(0)[0]["color"])
    mean = [(sum(x[k] for x in cols) + 2) // 5 for k in range(3)]
    assert (c & 255, (c >> 8) & 255, (c >> 16) & 255, c >> 24) == (mean[0], mean[1], mean[2], 200)
    # a capacity below the node's voxels filters nothing
    assert t.refine_colors([0], capacity=0) == (0, 0)


def test_deepen_known_answer():
    # Refinement's deepening: five points split the root (limit 4); child 1
    # (octant 0) keeps three. Deepening it splits it as doSplitting would
    # (remolod_octree.cu:303-400): ids 9..16, its points one level down by bit
    # 18 of the 20-bit coordinate, and a grid sampled at level 1, whose cell
    # is the 28-bit coordinate >> 20 (0.1 -> 25, 0.3 -> 76).
    t = unit_tree(max_points_per_node=4)
    cloud = pts([(0.1, 0.1, 0.1, 11), (0.3, 0.1, 0.1, 12), (0.1, 0.1, 0.3, 13),
                 (0.9, 0.9, 0.9, 14), (0.6, 0.2, 0.9, 15)])
    assert t.add_batch(cloud) == 0
    t.sweep()
    c1 = t.node(1)
    assert c1.is_leaf and c1.num_points == 3 and (c1.level, c1.X, c1.Y, c1.Z) == (1, 0, 0, 0)
    before = t.stats()
    refused, taken = t.deepen([1, 4], min_points=2)  # node 4 holds fewer than 2 points
    assert not refused and taken == 1
    t.sweep()
    s = t.stats()
    assert s.num_nodes == 17 and s.nodes_split == before.nodes_split + 1
    assert (s.batchlet_index, s.num_points_processed) == (before.batchlet_index, before.num_points_processed)
    c1 = t.node(1)
    assert not c1.is_leaf and list(c1.child) == list(range(9, 17)) and c1.num_points == 0
    # octants at level 1: (0.1,.1,.1) -> 0, (0.3,.1,.1) -> 4, (0.1,.1,.3) -> 1
    got = {k: list(t.leaf_points(9 + k)[1]) for k in range(8) if t.node(9 + k).num_points}
    assert got == {0: [0], 1: [2], 4: [1]}
    v = np.sort(t.node_voxels(1), order=["x", "y", "z"])
    cells = [(25, 25, 25, 11), (25, 25, 76, 13), (76, 25, 25, 12)]
    assert len(v) == 3
    for row, (cx, cy, cz, col) in zip(v, sorted(cells)):
        assert row["x"] == np.float32(0.5 * (cx + 0.5) / 128)
        assert row["y"] == np.float32(0.5 * (cy + 0.5) / 128)
        assert row["z"] == np.float32(0.5 * (cz + 0.5) / 128)
        assert row["color"] == col


def test_deepen_keeps_every_point_and_samples_the_deepened_nodes(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    t = ob.Tree(num_threads=4)
    t.reset(bmin, bmax)
    bs = cfg.batch_size
    for b in range(6):
        assert t.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    nodes = t.node_table()
    leaves = np.nonzero(nodes["is_leaf"] & (nodes["num_points"] > 0))[0]
    pick = leaves[np.argsort(-nodes["num_points"][leaves], kind="stable")][:12]
    before = t.stats()
    refused, taken = t.deepen(pick)
    assert not refused and taken == len(pick)
    for b in range(6, 8):
        assert t.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    t.sweep()
    s = t.stats()
    assert s.num_points == len(cloud) and s.dropped_points == 0 and s.overflow_flags == 0
    assert s.nodes_split >= before.nodes_split + len(pick)
    g = t.accumulate(8)
    assert g.sum_leaf_counts == len(cloud) and g.inner_with_sums == 0
    seen = np.zeros(len(cloud), dtype=np.int32)
    after = t.node_table()
    for i in np.nonzero(after["is_leaf"])[0]:
        seen[t.leaf_points(int(i))[1]] += 1
    assert np.all(seen == 1)
    for i in pick:
        assert after["is_leaf"][i] == 0 and after["num_voxels"][i] > 0
        assert after["num_voxels"][i] == int(sum(bin(int(w)).count("1") for w in t.node_grid(int(i))))


def twigs(nodes, limit=50000):
    """Nodes below the root whose eight children are all leaves, holding at
    most `limit` points together."""
    out = []
    for i in range(1, len(nodes)):
        kids = nodes["child"][i]
        if nodes["is_leaf"][i] or np.any(kids < 0):
            continue
        if np.all(nodes["is_leaf"][kids] == 1) and int(nodes["num_points"][kids].sum()) <= limit:
            out.append(i)
    return out


def test_collapse_merges_twigs_and_later_splits_reuse_their_grids(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    t = ob.Tree(num_threads=4)
    t.reset(bmin, bmax)
    bs = cfg.batch_size
    for b in range(6):
        assert t.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    t.sweep()
    # a normally built tree has no twig under the split limit (a node splits
    # only past it); deepened leaves are twigs: collapsing undoes deepening
    nodes = t.node_table()
    leaves = np.nonzero(nodes["is_leaf"] & (nodes["num_points"] > 0))[0]
    pick = [int(i) for i in leaves[np.argsort(-nodes["num_points"][leaves], kind="stable")][:10]]
    assert not twigs(nodes)
    held = {i: np.sort(t.leaf_points(i)[1]) for i in pick}
    assert t.deepen(pick) == (False, len(pick))
    t.sweep()
    nodes = t.node_table()
    cand = twigs(nodes)
    assert sorted(cand) == sorted(pick)
    before = t.stats()
    kids = {i: list(nodes["child"][i]) for i in cand}
    want = {i: int(nodes["num_points"][kids[i]].sum()) for i in cand}
    m, moved, dropped = t.collapse(cand + cand[:2])  # duplicates are ignored
    assert m == len(cand) and moved == sum(want.values())
    assert dropped == int(nodes["num_voxels"][cand].sum())
    t.sweep()
    s = t.stats()
    assert s.num_grids == before.num_grids - len(cand)
    after = t.node_table()
    for i in cand:
        assert after["is_leaf"][i] == 1 and after["num_points"][i] == want[i] and after["num_voxels"][i] == 0
        assert after["grid"][i] < 0
        assert np.array_equal(np.sort(t.leaf_points(i)[1]), held[i])
        assert np.all(after["num_points"][kids[i]] == 0)
    # every point still stored once, with its global index
    seen = np.zeros(6 * bs, dtype=np.int32)
    for i in np.nonzero(after["is_leaf"])[0]:
        seen[t.leaf_points(int(i))[1]] += 1
    assert np.all(seen == 1)
    g = t.accumulate(6)
    assert g.sum_leaf_counts == 6 * bs and g.inner_with_sums == 0
    # later batches split again and take the returned grids first
    grids_before = len(np.unique(after["grid"][after["grid"] >= 0]))
    for b in range(6, 8):
        assert t.add_batch(cloud[b * bs:(b + 1) * bs]) == 0
    t.sweep()
    s2 = t.stats()
    assert s2.num_points == len(cloud) and s2.dropped_points == 0
    fin = t.node_table()
    used = np.unique(fin["grid"][fin["grid"] >= 0])
    assert len(used) == s2.num_grids and len(used) >= grids_before
    seen = np.zeros(len(cloud), dtype=np.int32)
    for i in np.nonzero(fin["is_leaf"])[0]:
        seen[t.leaf_points(int(i))[1]] += 1
    assert np.all(seen == 1)


def test_collapse_known_answer_and_the_grid_pool():
    # The deepened child 1 of test_deepen_known_answer collapses back: a leaf
    # again with its three points, no voxels, its grid in the pool. Four more
    # points in its octant push it over the limit (4) and it splits again,
    # taking the pooled grid: no new grid, no new store charge for one.
    t = unit_tree(max_points_per_node=4)
    cloud = pts([(0.1, 0.1, 0.1, 11), (0.3, 0.1, 0.1, 12), (0.1, 0.1, 0.3, 13),
                 (0.9, 0.9, 0.9, 14), (0.6, 0.2, 0.9, 15)])
    assert t.add_batch(cloud) == 0
    assert t.deepen([1], min_points=2) == (False, 1)
    t.sweep()
    grids, offset = t.stats().num_grids, t.stats().persistent_offset
    assert t.collapse([1, 1, 0, 9]) == (1, 3, 3)  # the root and a leaf are not twigs
    t.sweep()
    s = t.stats()
    c1 = t.node(1)
    assert c1.is_leaf and c1.num_points == 3 and c1.num_voxels == 0 and c1.grid < 0
    assert sorted(t.leaf_points(1)[1]) == [0, 1, 2]
    assert s.num_grids == grids - 1 and s.num_nodes == 17
    more = pts([(0.2, 0.2, 0.2, 21), (0.2, 0.3, 0.2, 22), (0.3, 0.2, 0.3, 23), (0.1, 0.3, 0.3, 24)])
    assert t.add_batch(more) == 0
    t.sweep()
    s2 = t.stats()
    assert not t.node(1).is_leaf and t.node(1).grid >= 0
    assert s2.num_grids == grids  # the pooled grid, not a new one
    grid_bytes = 16 * ((128 ** 3 // 8 + 16) // 16)
    assert s2.persistent_offset - offset < grid_bytes  # no grid charge beyond the chunks


def test_deepen_is_refused_by_the_memory_check():
    # the batch's memory check (remolod_octree.cu:1181-1210) stops a deepening
    # pass too: nothing splits and the flag is raised
    # a margin of 1 byte (0 means the default 200 MB); the root grid and the
    # first batch's chunks take the store past 300,000 bytes
    t = unit_tree(max_points_per_node=4, persistent_capacity=300000, safety_margin=1)
    cloud = pts([(0.1, 0.1, 0.1, 11), (0.3, 0.1, 0.1, 12), (0.1, 0.1, 0.3, 13),
                 (0.9, 0.9, 0.9, 14), (0.6, 0.2, 0.9, 15)])
    assert t.add_batch(cloud) == 0
    t.sweep()
    n0 = t.stats().num_nodes
    assert t.stats().persistent_offset >= 300000
    assert t.deepen([1]) == (True, 0)
    t.sweep()
    assert t.stats().num_nodes == n0 and t.stats().mem_capacity_reached == 1
