"""Invariants of the oracle's deepening and collapsing on seeded random
clouds (small enough for the CPU suite): every point stays stored exactly
once with its global index, every node's voxel count is its grid's
population, grids in use are distinct and counted, no inner node holds sums,
and later batches build on the changed tree."""
import numpy as np
import pytest

from oracle import binding as ob

PT = ob.POINT_DTYPE


def cloud(rng, n, offset):
    centres = rng.random((6, 3))
    pick = rng.integers(0, 6, n)
    xyz = np.clip(centres[pick] + rng.normal(scale=0.05, size=(n, 3)), 0.0, 0.999)
    a = np.zeros(n, dtype=PT)
    a["x"], a["y"], a["z"] = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    a["color"] = (np.arange(n) + offset).astype(np.uint32) | 0xFF000000
    return a


def check(t, total):
    t.sweep()
    s = t.stats()
    assert s.dropped_points == 0 and s.overflow_flags == 0
    nodes = t.node_table()
    seen = np.zeros(total, dtype=np.int32)
    for i in np.nonzero(nodes["is_leaf"])[0]:
        seen[t.leaf_points(int(i))[1]] += 1
    assert np.all(seen == 1)
    grids = nodes["grid"][nodes["grid"] >= 0]
    assert len(np.unique(grids)) == len(grids) == s.num_grids
    for i in np.nonzero(nodes["grid"] >= 0)[0]:
        pop = int(np.unpackbits(t.node_grid(int(i)).view(np.uint8)).sum())
        # the root's grid is zeroed at its split while its earlier voxels stay
        # (remolod_octree.cu:372-387); every other grid starts empty at its split
        if i == 0:
            assert nodes["num_voxels"][i] >= pop
        else:
            assert nodes["num_voxels"][i] == pop, i
    g = t.accumulate(s.batchlet_index)
    assert g.sum_leaf_counts == total and g.inner_with_sums == 0
    return nodes


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_deepen_collapse_rounds_keep_the_invariants(seed):
    rng = np.random.default_rng(seed)
    t = ob.Tree(max_points_per_node=60, max_nodes=4000)
    t.reset((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    total = 0
    for rnd in range(4):
        assert t.add_batch(cloud(rng, 1500, total)) == 0
        total += 1500
        nodes = check(t, total)
        leaves = np.nonzero(nodes["is_leaf"] & (nodes["num_points"] >= 8))[0]
        pick = rng.choice(leaves, size=min(6, len(leaves)), replace=False)
        refused, taken = t.deepen(pick, min_points=8)
        assert not refused and taken == len(pick)
        nodes = check(t, total)
        twigs = [i for i in range(1, len(nodes)) if not nodes["is_leaf"][i]
                 and np.all(nodes["child"][i] >= 0) and np.all(nodes["is_leaf"][nodes["child"][i]] == 1)
                 and int(nodes["num_points"][nodes["child"][i]].sum()) <= 60]
        assert set(int(i) for i in pick) <= set(twigs)
        half = twigs[: (len(twigs) + 1) // 2]
        m, moved, _ = t.collapse(half)
        assert m == len(half)
        after = check(t, total)
        for i in half:
            assert after["is_leaf"][i] == 1 and after["grid"][i] < 0
