"""The synthetic generator: seeded, batch-reproducible, inside its box."""
import numpy as np

from remobench_b200 import synth


def test_batch_regenerates_alone():
    cfg = synth.config(1, num_points=4 * 4096, batch_size=4096, num_threads=3)
    full = synth.generate(cfg)
    one = synth.generate(cfg, first=2 * 4096, count=4096)
    assert np.array_equal(full[2 * 4096:3 * 4096].view(np.uint32), one.view(np.uint32))
    cfg1 = synth.config(1, num_points=4 * 4096, batch_size=4096, num_threads=1)
    assert np.array_equal(full.view(np.uint32), synth.generate(cfg1).view(np.uint32))


def test_seed_changes_cloud():
    a = synth.generate(synth.config(1, num_points=4096, batch_size=4096))
    b = synth.generate(synth.config(1, num_points=4096, batch_size=4096, seed=2))
    assert not np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_points_inside_box_and_scene_shape():
    cfg = synth.config(1, num_points=8 * 8192, batch_size=8192)
    p = synth.generate(cfg)
    lo, hi = synth.scene_box(cfg)
    xyz = np.stack([p["x"], p["y"], p["z"]], 1)
    assert np.all(xyz >= lo) and np.all(xyz <= hi)
    assert hi[0] == 200.0 and hi[1] == 200.0
    assert np.all((p["color"] >> 24) == 255)
    # scanline sensor: most points within 60 m of the lane at y = 100
    assert np.mean(np.abs(p["y"] - 100.0) < 60.0) > 0.8


def test_utm_float64_quantum():
    cfg = synth.config(3, num_points=4096, batch_size=4096)
    xyz, col = synth.generate_f64(cfg)
    assert np.all(xyz[:, 0] >= 500000.0) and np.all(xyz[:, 1] >= 4000000.0)
    mm = np.round(xyz * 1000.0)
    assert np.allclose(xyz * 1000.0, mm, atol=1e-3)
