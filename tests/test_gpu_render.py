"""Rasterize on the B200 against the CPU oracle: the pre-EDL 64-bit
depth|colour framebuffer bit-exact (LOD cut and flat), EDL within one colour
step per channel."""
import numpy as np
import pytest

from gpu_helpers import build_gpu, build_oracle
from oracle import binding as ob

pytestmark = pytest.mark.gpu

W, H = 1920, 1080  # configuration 1's view


def oracle_frame(f, cap=131072):
    o = ob.Frame()
    o.width, o.height = f.width, f.height
    for i in range(16):
        o.transform[i] = f.transform[i]
        o.transform_frozen[i] = f.transform_frozen[i]
    for a in range(3):
        o.box_min[a] = f.box_min[a]
        o.box_max[a] = f.box_max[a]
    o.lod_pixel_budget = f.lod_pixel_budget
    o.point_size = f.point_size
    o.drawlist_capacity = cap
    return o


@pytest.fixture(scope="module")
def c1_trees(c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size)
    tree = build_oracle(cloud, bmin, bmax, cfg.batch_size)
    return ctx, tree, bmin, bmax


@pytest.mark.parametrize("view", [dict(), dict(yaw=1.9, pitch=-0.35, radius_scale=0.35),
                                  dict(yaw=4.0, pitch=-1.2, radius_scale=0.15, budget=64.0),
                                  dict(point_size=3, radius_scale=0.5)])
def test_lod_framebuffer_bit_exact(c1_trees, view):
    import torch
    from remobench_b200.lod import make_frame
    ctx, tree, bmin, bmax = c1_trees
    view = dict(view)
    budget = view.pop("budget", 128.0)
    ps = view.pop("point_size", 1)
    f = make_frame(bmin, bmax, W, H, budget=budget, point_size=ps, **view)
    fb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    rgba = torch.empty(W * H, dtype=torch.int32, device="cuda")
    r = ctx.render(f, fb, rgba)
    ofb, orr, _ = tree.render(oracle_frame(f))
    g = fb.cpu().numpy().view(np.uint64)
    assert r.draw_items == orr.draw_items
    assert r.draw_samples == orr.draw_samples
    assert r.draw_items > 0
    assert np.array_equal(g, ofb)
    assert np.array_equal(rgba.cpu().numpy().view(np.uint32), (ofb & 0xFFFFFFFF).astype(np.uint32))


def test_flat_framebuffer_bit_exact(c1_cloud):
    import torch
    from remobench_b200.lod import Context, make_frame
    cfg, cloud, bmin, bmax = c1_cloud
    ctx = Context(pipeline=2)
    ctx.allocate(len(cloud), bmin, bmax)
    f = make_frame(bmin, bmax, W, H, radius_scale=0.6)
    dev = torch.from_numpy(cloud.view(np.float32).reshape(-1, 4)).cuda()
    fb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    r = ctx.render_flat(f, dev, fb)
    assert r.draw_samples == len(cloud)
    ofb = ob.render_flat(cloud, oracle_frame(f))
    assert np.array_equal(fb.cpu().numpy().view(np.uint64), ofb)


def test_edl_within_one_step(c1_trees):
    import torch
    from remobench_b200.lod import make_frame
    ctx, tree, bmin, bmax = c1_trees
    f = make_frame(bmin, bmax, W, H, edl=True, edl_strength=0.4)
    fb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    ctx.render(f, fb)
    ofb, _, _ = tree.render(oracle_frame(f))
    oe = ob.edl(ofb, W, H, 0.4)
    g = fb.cpu().numpy().view(np.uint64)
    assert np.array_equal(g >> 32, oe >> 32)  # depth untouched
    gc = (g & 0xFFFFFFFF).astype(np.uint32).view(np.uint8).reshape(-1, 4).astype(np.int32)
    oc = (oe & 0xFFFFFFFF).astype(np.uint32).view(np.uint8).reshape(-1, 4).astype(np.int32)
    assert np.max(np.abs(gc - oc)) <= 1  # libm vs CUDA log2f/expf: at most one 8-bit step


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_colour_modes_and_bounding_boxes_bit_exact(c1_trees, mode):
    """The reference viewer's colour modes (by node, by level, white;
    remo_draw.cuh:104-116) and its bounding-box wireframe drawn over the frame
    (remo_lines.cuh:120-137): the framebuffer with the boxes equals the
    oracle's render followed by its wireframe over the same draw items."""
    import torch
    from remobench_b200.lod import make_frame
    ctx, tree, bmin, bmax = c1_trees
    f = make_frame(bmin, bmax, W, H, yaw=0.8, pitch=-0.5, radius_scale=0.45)
    f.color_mode = mode
    f.show_bounding_box = 1
    fb = torch.empty(W * H, dtype=torch.int64, device="cuda")
    r = ctx.render(f, fb)
    of = oracle_frame(f)
    of.color_mode = mode
    ofb, orr, items = tree.render(of, item_nodes_cap=131072)
    assert r.draw_items == orr.draw_items > 0
    ofb = ob.wireframe(tree, of, ofb, items[:orr.draw_items])
    g = fb.cpu().numpy().view(np.uint64)
    assert np.array_equal(g, ofb)
    # the boxes drew something the points did not: line colours of the levels present
    f.show_bounding_box = 0
    fb2 = torch.empty(W * H, dtype=torch.int64, device="cuda")
    ctx.render(f, fb2)
    assert np.count_nonzero(fb2.cpu().numpy().view(np.uint64) != g) > 1000
