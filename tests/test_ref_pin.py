"""The CPU oracle against the reference itself: fixtures recorded by running
the reference's own kernels (kernels/remolod/*.cu, built from its sources by
oracle/ref/build_ref.py) on a B200 -- see tests/golden/make_ref_fixtures.py.

"ieee" is the reference built with its options minus fast math (and with
--fmad=false); the oracle must match it exactly on every structural field.
"shipped" is the reference's options verbatim (--use_fast_math); there the
approximate division may move points that sit within a couple of ulps of a
cell boundary, and the test bounds how much.
"""
import os

import numpy as np
import pytest

from oracle import binding as ob

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not present")
    return dict(np.load(path))


def mix64(v):
    v = v.astype(np.uint64)
    v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return v ^ (v >> np.uint64(31))


def multiset_digest(rows_u32):
    if len(rows_u32) == 0:
        return np.uint64(0)
    rows = rows_u32.astype(np.uint64)
    h = np.zeros(len(rows), dtype=np.uint64)
    with np.errstate(over="ignore"):
        for k in range(rows.shape[1]):
            h = mix64(h * np.uint64(0x100000001B3) + rows[:, k] + np.uint64(k + 1))
        return np.uint64(int(h.sum(dtype=np.uint64)))


def grid_digest(words):
    with np.errstate(over="ignore"):
        idx = np.arange(len(words), dtype=np.uint64)
        return np.uint64(int(mix64(words.astype(np.uint64) * np.uint64(2654435761) + idx).sum(dtype=np.uint64)))


def oracle_view(tree):
    nodes = tree.node_table()
    keys = np.stack([nodes["level"], nodes["X"], nodes["Y"], nodes["Z"]], 1).astype(np.int64)
    out = {"keys": keys, "counter": nodes["counter"].astype(np.int64),
           "num_points": nodes["num_points"].astype(np.int64), "num_voxels": nodes["num_voxels"].astype(np.int64),
           "is_leaf": nodes["is_leaf"].astype(bool), "has_grid": nodes["grid"] >= 0}
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
            p, _ = tree.leaf_points(i)
            pd[i] = multiset_digest(p.view(np.uint32).reshape(-1, 4))
        if nodes["num_voxels"][i]:
            v = tree.node_voxels(i)
            vd[i] = multiset_digest(v.view(np.uint32).reshape(-1, 4)[:, :3])
        g = tree.node_grid(i)
        if g is not None:
            gd[i] = grid_digest(g)
    out.update(point_digest=pd, voxel_digest=vd, grid_digest=gd)
    return out


def by_key(d):
    k = d["keys"]
    order = np.lexsort((k[:, 3], k[:, 2], k[:, 1], k[:, 0]))
    return {f: v[order] for f, v in d.items() if isinstance(v, np.ndarray) and v.shape[:1] == k.shape[:1]}


@pytest.fixture(scope="module")
def oracle_c1(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    t = ob.Tree()
    t.reset(bmin, bmax)
    bs = cfg.batch_size
    for b in range(8):
        t.add_batch(cloud[b * bs:(b + 1) * bs])
    t.sweep()
    t.accumulate(8)
    return t, oracle_view(t)


def test_same_input_cloud(c1_cloud):
    ref = load("ref_config1_ieee.npz")
    cloud = c1_cloud[1]
    assert multiset_digest(cloud.view(np.uint32).reshape(-1, 4)) == ref["input_digest"]


FIELDS = ["counter", "num_points", "num_voxels", "is_leaf", "has_grid", "child_keys", "point_digest",
          "voxel_digest", "grid_digest"]


def test_oracle_equals_reference_ieee_build(oracle_c1):
    t, ov = oracle_c1
    ref = load("ref_config1_ieee.npz")
    a, b = by_key(ov), by_key(ref)
    assert np.array_equal(a["keys"], b["keys"])
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    s = t.stats()
    assert s.num_nodes == ref["stats_numNodes"]
    assert s.num_inner == ref["stats_numInner"] and s.num_leaves == ref["stats_numLeaves"]
    assert s.num_points == ref["stats_numPoints"] and s.num_voxels == ref["stats_numVoxels"]
    assert s.persistent_offset == ref["stats_allocatedBytes_persistent"]
    assert s.num_chunks_points == ref["stats_numChunksPoints"]
    assert s.num_chunks_voxels == ref["stats_numChunksVoxels"]
    assert s.chunk_pool_size == ref["stats_chunkPoolSize"]
    assert s.num_allocated_chunks == ref["stats_numAllocatedChunks"]


def test_oracle_fp64_accumulate_equals_reference(oracle_c1):
    t, ov = oracle_c1
    ref = load("ref_config1_ieee.npz")
    nodes = t.node_table()
    keys = ov["keys"]
    rk = {tuple(k): i for i, k in enumerate(ref["keys"])}
    for i in range(len(nodes)):
        j = rk[tuple(keys[i])]
        a = t.accum_f(i)
        assert a.count == ref["accum_count"][j]
        # FP64 sums depend on fold order (block reduction vs sequential): relative 1e-12
        assert np.allclose(np.array(a.g), ref["accum_g"][j], rtol=1e-12, atol=1e-9)


def test_oracle_framebuffer_equals_reference(oracle_c1):
    t, _ = oracle_c1
    ref = load("ref_config1_ieee.npz")
    frames = ref["frames"]
    for k in range(len(frames)):
        f = ob.Frame()
        f.width, f.height = 480.0, 270.0
        for i, v in enumerate(frames[k].reshape(-1)):
            f.transform[i] = float(v)
            f.transform_frozen[i] = float(v)
        from remobench_b200 import synth
        lo, hi = synth.scene_box(synth.config(1))
        for a in range(3):
            f.box_min[a] = float(lo[a])
            f.box_max[a] = float(hi[a])
        f.lod_pixel_budget = 128.0
        f.point_size = 1
        f.drawlist_capacity = 131072
        fb, _, _ = t.render(f)
        rfb = ref["fb"][k]
        # depth (high 32 bits) is exact; a voxel's colour is first-come in the reference
        assert np.array_equal(fb >> np.uint64(32), rfb >> np.uint64(32))
        same = np.mean(fb == rfb)
        assert same > 0.9, same


def test_truncation_equals_reference():
    ref = load("ref_config1_ieee_store230MB.npz")
    from remobench_b200 import synth
    cfg = synth.config(1)
    cloud = synth.generate(cfg)
    bmin, bmax = synth.scene_box(cfg)
    t = ob.Tree(persistent_capacity=int(ref["persistent_capacity"]))
    t.reset(bmin, bmax)
    bs = cfg.batch_size
    done = 0
    for b in range(8):
        if t.add_batch(cloud[b * bs:(b + 1) * bs]) != 0:
            break
        done += 1
    t.sweep()
    s = t.stats()
    assert done == ref["stats_batchletIndex"] == 5
    assert s.mem_capacity_reached == ref["stats_memCapacityReached"] == 1
    assert s.num_nodes == ref["stats_numNodes"]
    assert s.num_voxels == ref["stats_numVoxels"]
    assert s.persistent_offset == ref["stats_allocatedBytes_persistent"]
    ov = by_key(oracle_view(t))
    rv = by_key(ref)
    for f in ["counter", "num_points", "num_voxels", "point_digest", "grid_digest"]:
        assert np.array_equal(ov[f], rv[f]), f


def test_oracle_vs_shipped_fast_math_build(oracle_c1):
    """The reference as shipped divides with fast math, which could move a point
    lying within a couple of ulps of a cell boundary. On this cloud none moves:
    the tree is identical field for field."""
    t, ov = oracle_c1
    ref = load("ref_config1_shipped.npz")
    a, b = by_key(ov), by_key(ref)
    assert np.array_equal(a["keys"], b["keys"])
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
    assert ref["stats_numPoints"] == t.stats().num_points
    assert ref["stats_allocatedBytes_persistent"] == t.stats().persistent_offset
