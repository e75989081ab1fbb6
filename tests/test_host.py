"""The C++ host layer (ILodPipeline, PipelineRegistry, PointSource, the
headless harness).

CPU: the registry's gate decisions against figures worked by hand from
src/shell/PipelineRegistry.cpp:54-250 and the pipelines' PipelineInfo
(src/pipelines/RemolodPipeline.cpp:23-61, SimlodPipeline.cpp:28-62,
FlatPipeline.cpp:22-35); the harness's option handling.
GPU: the harness's frame loop (render -> pump -> build) yields the oracle's
tree and framebuffer for the same cloud and view, for each pipeline and across
a pipeline switch.
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "remobench_b200", "lib")
HARNESS = os.path.join(LIB, "rb_harness")

MIB = 1 << 20
RING_50 = 50 * 1_000_000 * 16                         # 800 MB: fifty 1M-point slots of 16 B points
REMOLOD_FIXED = 512 * MIB + 200_000 * (152 + 112)      # momentary buffer + node pool + accumulators
SIMLOD_FIXED = 512 * MIB + 200_000 * 152
MIN_STORE = 512 * MIB
MARGIN = 200_000_000


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    from remobench_b200 import build
    build.build_host()
    exe = str(tmp_path_factory.mktemp("host") / "probe")
    src = os.path.join(ROOT, "tests", "host_registry_probe.cpp")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(ROOT, "remobench_b200", "host"), "-I",
                           os.path.join(ROOT, "remobench_b200", "csrc"), "-o", exe, src, "-L", LIB, "-lrb_host",
                           "-lrb_cuda", "-lrb_synth", "-Wl,-rpath," + LIB])
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    kv = {}
    for line in out.splitlines():
        k, _, v = line.partition(" ")
        kv[k] = v
    return kv


def test_registration(probe):
    assert probe["registered"] == "4"  # duplicate id and null factory refused
    assert probe["info.remolod"] == f"RemoLOD 1 0 50 48.0 26.0 {MIN_STORE} {REMOLOD_FIXED}"
    assert probe["info.simlod"] == f"SimLOD 1 0 50 48.0 26.0 {MIN_STORE} {SIMLOD_FIXED}"
    assert probe["info.flat"] == "Flat 0 1 0 0.0 0.0 0 0"


def test_gate_streaming_partial_tree(probe):
    # 100M points in a 3 GB budget: runs, truncates at the predicted fraction
    p = "remolod_100M_3GB"
    assert int(probe[p + ".input"]) == RING_50
    assert int(probe[p + ".min_required"]) == 26 * 100_000_000 + RING_50 + REMOLOD_FIXED
    assert int(probe[p + ".floor"]) == MIN_STORE + RING_50 + REMOLOD_FIXED
    assert probe[p + ".fits"] == "1"
    usable = (3_000_000_000 - RING_50 - REMOLOD_FIXED) - MARGIN
    assert abs(float(probe[p + ".predicted"]) - usable / 26 / 100_000_000) < 1e-8
    assert probe[p + ".warning"].startswith("predicted to take in about 54% of the cloud")
    need_gb = (26 * 100_000_000 + RING_50 + REMOLOD_FIXED) / 1e9
    assert f"needs a {need_gb:.1f} GB budget" in probe[p + ".warning"]
    assert probe[p + ".reason"] == ""


def test_gate_refusal_below_floor(probe):
    p = "remolod_100M_1.9GB"
    assert probe[p + ".fits"] == "0"
    floor_gb = (MIN_STORE + RING_50 + REMOLOD_FIXED) / 1e9
    reason = probe[p + ".reason"]
    assert reason.startswith("refused: the budget is 1.9 GB, below this pipeline's floor of "
                             f"{floor_gb:.1f} GB (a 0.8 GB ring, 0.59 GB of fixed buffers")
    assert "smallest store" in reason
    assert probe["switch_refused"].startswith("0 RemoLOD: refused: the budget is 0.0 GB")


def test_gate_whole_fit_and_flat(probe):
    assert probe["simlod_1B_180GB.predicted"] == "1.000000000"
    assert probe["simlod_1B_180GB.warning"] == ""
    # flat cannot truncate: its floor is the resident cloud itself
    assert int(probe["flat_100M_1.5GB.floor"]) == 16 * 100_000_000
    assert probe["flat_100M_1.5GB.fits"] == "0"
    assert probe["flat_100M_1.5GB.reason"].startswith("refused: the whole cloud (100000000 points) needs 1.6 GB")
    assert "cannot stop on a partial tree" in probe["flat_100M_1.5GB.reason"]
    assert probe["flat_100M_2GB.fits"] == "1"
    assert probe["flat_100M_2GB.predicted"] == "1.000000000"


def test_gate_small_cloud_prediction_kept(probe):
    # The prediction sizes the store at 48 B/pt without allocate()'s 512 MB floor,
    # so a 2M-point cloud is predicted 0% although it completes; kept as the reference has it.
    assert probe["remolod_2M_8GB.fits"] == "1"
    assert probe["remolod_2M_8GB.predicted"] == "0.000000000"
    assert int(probe["remolod_2M_8GB.input"]) == 2 * 16_000_000  # ring no deeper than the cloud


def test_resident_ceiling(probe):
    assert "reaches only the first 50M points of this 60M-point cloud" in probe["resident_60M_100GB.reason"]
    assert probe["resident_40M_100GB.reason"] == ""


def test_switch_errors(probe):
    assert probe["switch_unknown"] == "0 unknown pipeline: nonesuch"
    assert probe["reload_inactive"] == "0 no active pipeline"


def test_harness_cli_without_device():
    from remobench_b200 import build
    build.build_host()
    r = subprocess.run([HARNESS, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown option --bogus" in r.stderr
    r = subprocess.run([HARNESS, "--size", "0", "10"], capture_output=True, text=True)
    assert r.returncode == 2


# ---------------------------------------------------------------- GPU


def _run_harness(tmp_path, *args, frame=None, timeout=600):
    cmd = [HARNESS] + [str(a) for a in args]
    if frame is not None:
        fpath = tmp_path / "uniforms.bin"
        fpath.write_bytes(bytes(frame))
        cmd += ["--frame-file", str(fpath)]
    surf = tmp_path / "surface.bin"
    cmd += ["--surface-out", str(surf)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    lines = [line for line in r.stdout.splitlines() if line.startswith("{")]
    assert lines, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    summary = json.loads(lines[-1])
    rgba = np.fromfile(surf, dtype=np.uint32) if surf.exists() else None
    return r.returncode, summary, rgba, r


def _oracle_frame(f):
    from oracle import binding as ob
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
    o.drawlist_capacity = 131072
    return o


W, H = 960, 540


@pytest.fixture(scope="module")
def c1_oracle(c1_cloud):
    from gpu_helpers import build_oracle
    cfg, cloud, bmin, bmax = c1_cloud
    return build_oracle(cloud, bmin, bmax, cfg.batch_size)


@pytest.mark.gpu
@pytest.mark.parametrize("pipeline", ["remolod", "simlod"])
def test_harness_progressive_matches_oracle(tmp_path, c1_cloud, c1_oracle, pipeline):
    from remobench_b200.lod import make_frame
    cfg, cloud, bmin, bmax = c1_cloud
    f = make_frame(bmin, bmax, W, H, yaw=1.2, pitch=-0.5, radius_scale=0.6)
    rc, s, rgba, r = _run_harness(tmp_path, "--pipeline", pipeline, "--config", 1, "--seed", cfg.seed,
                                  "--size", W, H, frame=f)
    assert rc == 0, r.stderr
    st = c1_oracle.stats()
    assert s["pipeline"] == pipeline and s["ok"]
    assert s["cloud_points"] == len(cloud) == s["points_ingested"]
    assert (s["nodes"], s["inner"], s["leaves"]) == (st.num_nodes, st.num_inner, st.num_leaves)
    assert (s["points"], s["voxels"]) == (st.num_points, st.num_voxels)
    assert s["max_points_per_node"] == st.max_points_per_node
    assert not s["overran_consumer"] and not s["mem_capacity_reached"]
    assert s["build_launches"] > 0 and s["build_ms"] > 0
    ofb, orr, _ = c1_oracle.render(_oracle_frame(f))
    assert s["visible_nodes"] == orr.draw_items
    assert s["visible_samples"] == orr.draw_samples
    assert np.array_equal(rgba, (ofb & 0xFFFFFFFF).astype(np.uint32))


@pytest.mark.gpu
def test_harness_flat_matches_oracle(tmp_path, c1_cloud):
    from oracle import binding as ob
    from remobench_b200.lod import make_frame
    cfg, cloud, bmin, bmax = c1_cloud
    f = make_frame(bmin, bmax, W, H, radius_scale=0.7)
    rc, s, rgba, r = _run_harness(tmp_path, "--pipeline", "flat", "--config", 1, "--seed", cfg.seed,
                                  "--size", W, H, frame=f)
    assert rc == 0, r.stderr
    assert s["visible_samples"] == len(cloud)
    ofb = ob.render_flat(cloud, _oracle_frame(f))
    assert np.array_equal(rgba, (ofb & 0xFFFFFFFF).astype(np.uint32))


@pytest.mark.gpu
def test_harness_switch_and_dump(tmp_path, c1_cloud, c1_oracle):
    # simlod for two frames, then remolod from batch 0 on the re-started ring
    cfg, cloud, bmin, bmax = c1_cloud
    ppm = tmp_path / "frame.ppm"
    rc, s, rgba, r = _run_harness(tmp_path, "--pipeline", "simlod", "--switch-to", "remolod", "--switch-after", 2,
                                  "--config", 1, "--seed", cfg.seed, "--size", 320, 180, "--dump-frame", ppm,
                                  "--trace")
    assert rc == 0, r.stderr
    st = c1_oracle.stats()
    assert s["pipeline"] == "remolod"
    assert (s["nodes"], s["points"], s["voxels"]) == (st.num_nodes, st.num_points, st.num_voxels)
    trace = [json.loads(line) for line in r.stdout.splitlines() if line.startswith('{"frame"')]
    assert [t["pipeline"] for t in trace[:2]] == ["simlod", "simlod"]
    assert trace[2]["pipeline"] == "remolod" and trace[2]["pointsIngested"] == 0  # reset frame
    head = ppm.read_bytes()[:15]
    assert head.startswith(b"P6\n320 180\n255\n")
    assert "rb_harness: pipeline=remolod" in r.stdout and "remolod.construct" in r.stdout


@pytest.mark.gpu
def test_harness_refuses_small_budget(tmp_path, c1_cloud):
    cfg, cloud, bmin, bmax = c1_cloud
    rc, s, _, r = _run_harness(tmp_path, "--pipeline", "remolod", "--config", 1, "--seed", cfg.seed,
                               "--device-budget", 0.5, "--size", 64, 64)
    assert rc == 1
    assert not s["ok"] and s["refused"].startswith("RemoLOD: refused: the budget is 0.5 GB")
