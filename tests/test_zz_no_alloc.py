"""rb_render_noalloc, the render entry point that allocates nothing.

It serves callers that build the tree ahead of time but render from a place
where they cannot allocate -- a real-time frame callback that may not take the
allocator's lock or risk an allocation failure mid-frame, or an embedder whose
own pool holds all device memory after start-up. Its scratch is a static device
array shared by every call, so this test renders twice in a row through the
C ABI, with different views, and checks each frame against rb_render's: the
second call must not see the first call's flags, draw list or counters. The file
runs last so that a failure here leaves every other test already run; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from remobench_b200 import capi

pytestmark = pytest.mark.gpu

W, H = 960, 540


@pytest.fixture(scope="module")
def small_tree():
    from remobench_b200 import synth
    from remobench_b200.lod import Context, DeviceRing
    cfg = synth.config(1, num_points=4 * 131072, batch_size=131072)
    pts = synth.generate(cfg)
    bmin, bmax = synth.scene_box(cfg)
    ctx = Context(slot_capacity=cfg.batch_size, time_budget_ms=0.0, max_points_per_node=20000)
    ctx.allocate(len(pts), bmin, bmax)
    ring = DeviceRing(pts, cfg.batch_size, slots=ctx.cfg.ring_slots, slot_capacity=cfg.batch_size)
    ring.upload_window(0)
    r = ctx.build(ring.ring, ring.sizes, ring.uploaded, ring.num_batches)
    assert r.batches_consumed == 4
    return ctx, bmin, bmax


def render_noalloc(ctx, frame, fb, rgba):
    r = capi.RenderResult()
    st = capi.lib().rb_render_noalloc(ctx.h, ctypes.byref(frame), fb.data_ptr(), rgba.data_ptr(), 0,
                                      ctypes.byref(r))
    assert st == capi.RB_OK, capi.lib().rb_last_error(ctx.h)
    return r


@pytest.mark.parametrize("edl", [False, True])
def test_noalloc_render_matches_rb_render_twice_in_a_row(small_tree, edl):
    import torch
    from remobench_b200.lod import make_frame
    ctx, bmin, bmax = small_tree
    views = [dict(), dict(yaw=2.4, pitch=-0.4, radius_scale=0.3, budget=48.0)]
    for view in views:
        view = dict(view)
        budget = view.pop("budget", 128.0)
        f = make_frame(bmin, bmax, W, H, budget=budget, edl=edl, **view)
        fb_ref = torch.empty(W * H, dtype=torch.int64, device="cuda")
        rgba_ref = torch.empty(W * H, dtype=torch.int32, device="cuda")
        fb = torch.full((W * H,), 7, dtype=torch.int64, device="cuda")
        rgba = torch.full((W * H,), 7, dtype=torch.int32, device="cuda")
        ref = ctx.render(f, fb_ref, rgba_ref)
        got = render_noalloc(ctx, f, fb, rgba)
        assert got.draw_items == ref.draw_items > 0
        assert got.draw_samples == ref.draw_samples
        assert got.drawlist_overflow == ref.drawlist_overflow == 0
        # bit-exact, the tolerance of the render parity tests
        assert torch.equal(fb, fb_ref)
        assert torch.equal(rgba, rgba_ref)


def test_noalloc_render_takes_no_device_memory(small_tree):
    """The claim itself: after one warm-up call (which only settles the
    caching of torch's own tensors below), EDL-on renders leave the device's
    free memory unchanged: no call allocates, whatever the frame size."""
    import torch
    from remobench_b200.lod import make_frame
    ctx, bmin, bmax = small_tree
    w, h = 1920, 1080
    fb = torch.empty(w * h, dtype=torch.int64, device="cuda")
    rgba = torch.empty(w * h, dtype=torch.int32, device="cuda")
    f = make_frame(bmin, bmax, w, h, edl=True)
    render_noalloc(ctx, f, fb, rgba)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for yaw in (0.3, 1.1, 2.0):
        render_noalloc(ctx, make_frame(bmin, bmax, w, h, yaw=yaw, edl=True), fb, rgba)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_contexts_beyond_its_limit():
    from remobench_b200 import synth
    from remobench_b200.lod import Context, make_frame
    import torch
    cfg = synth.config(1, num_points=65536, batch_size=65536)
    bmin, bmax = synth.scene_box(cfg)
    ctx = Context(slot_capacity=65536, max_nodes=300000)
    ctx.allocate(65536, bmin, bmax)
    f = make_frame(bmin, bmax, 64, 64)
    fb = torch.empty(64 * 64, dtype=torch.int64, device="cuda")
    r = capi.RenderResult()
    st = capi.lib().rb_render_noalloc(ctx.h, ctypes.byref(f), fb.data_ptr(), 0, 0, ctypes.byref(r))
    assert st == capi.RB_ERR_CAPACITY
    assert b"262144" in capi.lib().rb_last_error(ctx.h)
