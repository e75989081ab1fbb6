""".simlod files (src/io/RawReader.h:10-16, RawReader.cpp): the Python writer
and reader against the C++ host's reader, the reference's size rules, and, on
the GPU, the headless harness streaming a .simlod file from disk into the same
tree the oracle builds from the same points."""
import os
import subprocess

import numpy as np
import pytest

from remobench_b200 import simlod

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "remobench_b200", "lib")
HOST = os.path.join(ROOT, "remobench_b200", "host")


def fnv64(pts):
    h = 1469598103934665603
    for w in np.ascontiguousarray(pts).view(np.uint32):
        h = ((h ^ int(w)) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("simlod") / "probe")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", HOST, "-o", exe,
                           os.path.join(ROOT, "tests", "host_simlod_probe.cpp"), os.path.join(HOST, "simlod_file.cpp")])
    return exe


def run_probe(exe, path):
    out = subprocess.run([exe, path], capture_output=True, text=True).stdout
    return {k: v for k, _, v in (line.partition(" ") for line in out.splitlines())}


def small_cloud(n=5000, seed=3):
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=simlod.POINT_DTYPE)
    p["x"] = rng.uniform(500000.0, 500300.0, n).astype(np.float32)
    p["y"] = rng.uniform(4000000.0, 4000200.0, n).astype(np.float32)
    p["z"] = rng.uniform(10.0, 60.0, n).astype(np.float32)
    p["color"] = rng.integers(0, 2**32, n, dtype=np.uint32)
    return p


def test_roundtrip_and_cpp_reader_agree(tmp_path, probe):
    pts = small_cloud()
    path = str(tmp_path / "c.simlod")
    # a header box that is wrong on purpose: the reader uses the observed one
    simlod.write(path, pts, header_box=[0, 0, 0, 1, 1, 1])
    n, box = simlod.header(path)
    assert n == len(pts) and list(box) == [0, 0, 0, 1, 1, 1]
    assert np.array_equal(np.array(simlod.points(path)), pts)
    loaded, bmin, bmax = simlod.load(path)
    b = simlod.bounds(path)
    kv = run_probe(probe, path)
    assert int(kv["points"]) == len(pts)
    assert [float(v) for v in kv["bounds"].split()] == list(b)
    assert int(kv["digest"]) == fnv64(loaded)
    assert kv["past_end"] == "0"
    # translated to the observed minimum: the box starts at 0
    assert float(loaded["x"].min()) == 0.0 and float(loaded["y"].min()) == 0.0
    assert np.allclose(bmax, b[3:] - b[:3])


def test_size_rules(tmp_path, probe):
    short = tmp_path / "short.simlod"
    short.write_bytes(b"\0" * 20)
    ragged = tmp_path / "ragged.simlod"
    ragged.write_bytes(b"\0" * (24 + 17))
    empty = tmp_path / "empty.simlod"
    empty.write_bytes(b"\0" * 24)
    for path, words in ((short, "shorter"), (ragged, "whole number"), (empty, "no points")):
        with pytest.raises(ValueError, match=words):
            simlod.header(str(path))
        assert words in run_probe(probe, str(path)).get("error", "")


@pytest.mark.gpu
def test_harness_streams_a_simlod_file(tmp_path, c1_cloud):
    """Configuration 1 written as a .simlod file (world coordinates, a UTM-like
    offset) and streamed from disk by the harness: the tree equals the oracle's
    on the points the reader yields."""
    import json
    from gpu_helpers import build_oracle
    cfg, cloud, bmin, bmax = c1_cloud
    world = cloud.copy()
    world["x"] += np.float32(1000.0)
    world["y"] += np.float32(2000.0)
    path = str(tmp_path / "c1.simlod")
    simlod.write(path, world)
    pts, lo, hi = simlod.load(path)
    tree = build_oracle(pts, lo, hi, cfg.batch_size)
    r = subprocess.run([os.path.join(LIB, "rb_harness"), "--pipeline", "remolod", "--file", path, "--batch",
                        str(cfg.batch_size), "--size", "320", "180"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    s = json.loads([line for line in r.stdout.splitlines() if line.startswith("{")][-1])
    st = tree.stats()
    assert s["cloud_points"] == len(cloud) == s["points_ingested"]
    assert (s["nodes"], s["points"], s["voxels"]) == (st.num_nodes, st.num_points, st.num_voxels)
