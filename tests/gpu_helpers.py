"""Shared helpers of the GPU parity tests: build the same cloud through the
CUDA path (C ABI) and through the CPU oracle, and compare them."""
import numpy as np

from oracle import binding as ob


def build_gpu(cloud, bmin, bmax, batch_size, budget=0, per_call=20, **cfg):
    from remobench_b200.lod import Context, DeviceRing
    slot_cap = cfg.pop("slot_capacity", batch_size)
    cfg.setdefault("time_budget_ms", 0.0)
    ctx = Context(slot_capacity=slot_cap, max_batches_per_build=per_call, **cfg)
    ctx.allocate(len(cloud), bmin, bmax, budget)
    ring = DeviceRing(cloud, batch_size, slots=ctx.cfg.ring_slots, slot_capacity=slot_cap)
    consumed, calls = 0, 0
    while consumed < ring.num_batches:
        ring.upload_window(consumed)
        r = ctx.build(ring.ring, ring.sizes, ring.uploaded, ring.num_batches)
        calls += 1
        if r.batches_this_call == 0:
            break
        consumed = r.batches_consumed
    return ctx, calls


def build_oracle(cloud, bmin, bmax, batch_size, **cfg):
    t = ob.Tree(**cfg)
    t.reset(bmin, bmax)
    for b in range((len(cloud) + batch_size - 1) // batch_size):
        if t.add_batch(cloud[b * batch_size:(b + 1) * batch_size]) != 0:
            break
    t.sweep()
    return t


NODE_FIELDS = ["counter", "num_points", "level", "X", "Y", "Z", "num_voxels", "num_point_chunks",
               "num_voxel_chunks", "is_leaf"]


def compare_nodes(ctx, tree):
    g = ctx.nodes()
    o = tree.node_table()
    assert len(g) == len(o), (len(g), len(o))
    assert np.array_equal(g["child"], o["child"])
    for f in NODE_FIELDS:
        assert np.array_equal(g[f], o[f]), f
    assert np.array_equal(g["has_grid"], (o["grid"] >= 0).astype(np.uint32))
    return g


def _rows(a):
    return a.view(np.uint32).reshape(-1, 4)


def compare_points(ctx, tree, nodes):
    for i in np.nonzero(nodes["num_points"])[0]:
        i = int(i)
        gp, gi = ctx.node_points(i)
        op, oi = tree.leaf_points(i)
        assert len(gp) == len(op), i
        a, b = np.argsort(gi, kind="stable"), np.argsort(oi, kind="stable")
        assert np.array_equal(gi[a], oi[b]), i
        assert np.array_equal(_rows(gp)[a], _rows(op)[b]), i


def compare_voxels(ctx, tree, nodes, colours=True):
    for i in np.nonzero(nodes["num_voxels"])[0]:
        i = int(i)
        gv = _rows(ctx.node_voxels(i))
        ov = _rows(tree.node_voxels(i))
        assert len(gv) == len(ov), i
        if not colours:
            gv, ov = gv[:, :3], ov[:, :3]
        ga = gv[np.lexsort(gv.T[::-1])]
        oa = ov[np.lexsort(ov.T[::-1])]
        assert np.array_equal(ga, oa), i


def compare_grids(ctx, tree, nodes):
    for i in np.nonzero(nodes["has_grid"])[0]:
        i = int(i)
        assert np.array_equal(ctx.node_grid(i), tree.node_grid(i)), i


STAT_FIELDS = ["num_points", "num_voxels", "num_inner", "num_leaves", "num_nonempty_leaves",
               "num_chunks_points", "num_chunks_voxels", "batchlet_index", "num_allocated_chunks",
               "chunk_pool_size", "mem_capacity_reached", "counter_underflows", "dropped_points",
               "nodes_split", "spilled_points", "num_grids", "overflow_flags", "max_points_per_node"]


def compare_stats(ctx, tree):
    g = ctx.stats()
    o = tree.stats()
    for f in STAT_FIELDS:
        assert getattr(g, f) == getattr(o, f), (f, getattr(g, f), getattr(o, f))
    assert g.num_nodes == o.num_nodes
    assert g.persistent_offset == o.persistent_offset
    assert g.num_points_ingested == o.num_points_processed
    return g


def compare_accums(ctx, tree):
    ga = ctx.accums()
    for i in range(tree.num_nodes()):
        a = tree.accum_i(i)
        g = ga[i]
        assert list(g["s1"]) == list(a.s1), i
        assert list(g["s2_lo"]) == list(a.s2_lo), i
        assert list(g["s2_hi"]) == list(a.s2_hi), i
        assert list(g["c1"]) == list(a.c1), i
        assert list(g["c2"]) == list(a.c2), i
        assert g["count"] == a.count, i


def quant28(coord, mn, size):
    """The 28-bit octree coordinate of remolod_octree.cu:167-169 in IEEE float32
    arithmetic (subtract, scale by 2^28 -- exact --, divide), converted with
    saturating round-toward-zero as the CUDA path's __float2uint_rz."""
    d = np.asarray(coord, dtype=np.float32) - np.float32(mn)
    q = (np.float32(268435456.0) * d) / np.float32(size)
    q = np.where(np.isnan(q) | (q < 0), np.float32(0), q).astype(np.float64)
    return np.minimum(np.floor(q), 4294967295.0).astype(np.int64)


def mix64(v):
    v = np.asarray(v).astype(np.uint64)
    with np.errstate(over="ignore"):
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return v ^ (v >> np.uint64(31))


def gpu_view(ctx):
    """The GPU tree in the fixture format of tests/golden/make_ref_fixtures.py:
    nodes keyed by (level, X, Y, Z) with order-independent digests of their
    point multisets, voxel positions and occupancy grids."""
    from test_ref_pin import grid_digest, multiset_digest
    nodes = ctx.nodes()
    keys = np.stack([nodes["level"], nodes["X"], nodes["Y"], nodes["Z"]], 1).astype(np.int64)
    out = {"keys": keys, "counter": nodes["counter"].astype(np.int64),
           "num_points": nodes["num_points"].astype(np.int64), "num_voxels": nodes["num_voxels"].astype(np.int64),
           "is_leaf": nodes["is_leaf"].astype(bool), "has_grid": nodes["has_grid"].astype(bool)}
    nn = len(nodes)
    ckeys = np.full((nn, 8, 4), -1, dtype=np.int64)
    for c in range(8):
        m = nodes["child"][:, c] >= 0
        ckeys[m, c] = keys[nodes["child"][m, c]]
    out["child_keys"] = ckeys
    pd = np.zeros(nn, dtype=np.uint64)
    vd = np.zeros(nn, dtype=np.uint64)
    gd = np.zeros(nn, dtype=np.uint64)
    for i in range(nn):
        if nodes["is_leaf"][i] and nodes["num_points"][i]:
            p, _ = ctx.node_points(i)
            pd[i] = multiset_digest(p.view(np.uint32).reshape(-1, 4))
        if nodes["num_voxels"][i]:
            v = ctx.node_voxels(i)
            vd[i] = multiset_digest(v.view(np.uint32).reshape(-1, 4)[:, :3])
        if nodes["has_grid"][i]:
            gd[i] = grid_digest(ctx.node_grid(i))
    out.update(point_digest=pd, voxel_digest=vd, grid_digest=gd)
    return out
