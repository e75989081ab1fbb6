"""The quality harness (remobench_b200/quality.py) on configuration 1: at a
pixel budget so small that the LOD cut opens every node down to its leaves,
the LOD render is the flat render bit for bit (every point drawn, no voxel),
so PSNR is infinite and coverage complete; as the budget grows, voxels stand
in for points and the image drifts from the flat ground truth."""
import numpy as np
import pytest

from gpu_helpers import build_gpu

pytestmark = pytest.mark.gpu

W, H = 960, 540


def test_lod_converges_to_flat(c1_cloud):
    import torch
    from remobench_b200 import capi, quality
    from remobench_b200.lod import Context, make_frame
    cfg, cloud, bmin, bmax = c1_cloud
    ctx, _ = build_gpu(cloud, bmin, bmax, cfg.batch_size)
    flat = Context(pipeline=capi.RB_PIPELINE_FLAT)
    flat.allocate(len(cloud), bmin, bmax)
    dev = torch.from_numpy(cloud.view(np.float32).reshape(-1, 4)).cuda()
    view = dict(yaw=0.9, pitch=-0.45, radius_scale=0.5)
    tiny = quality.compare(ctx, flat, dev, make_frame(bmin, bmax, W, H, budget=1e-6, **view))
    assert tiny["psnr"] == float("inf") and tiny["coverage"] == 1.0 and tiny["depth_rel_rmse"] == 0.0
    # budgets up to a few pixels still open every node on this view (the
    # render is exact); coarser cuts draw voxels and drift from the flat image
    psnrs = [quality.compare(ctx, flat, dev, make_frame(bmin, bmax, W, H, budget=b, **view))["psnr"]
             for b in (8.0, 64.0, 512.0)]
    assert all(a >= b for a, b in zip(psnrs, psnrs[1:])), psnrs
    assert np.isfinite(psnrs[-1]) and psnrs[-1] < 40.0, psnrs
