"""Benchmark of the progressive LOD hot path on B200.

Workload (configuration 2): a 100M-point synthetic lidar cloud (2 x 2 km tile,
2,000 boxes, 20,000 poles, seeded), streamed in 1M-point batches through
Update + Accumulate (20 batches per build call, Accumulate after each, as the
reference's frame loop does: src/pipelines/RemolodPipeline.cpp:296-438), then
rasterized at 3840x2160 along a seeded orbit.

One step = reset + ingest of the whole cloud. `value` is ingest Mpts/s with the
cloud resident in HBM (CUDA events on the launching stream, max over ranks);
`e2e` is the same through rb_ingest_host from pinned host memory, host->device
copies inside the timed region. Inputs (1.6 GB) are larger than L2 (126 MB).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank ingests its own seeded cloud: replicas, no
collective on the data path (the reference is single-GPU).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ingest Mpts/s (Update+Accumulate) + raster ms/frame"
UNIT = "Mpts/s"
BATCH = 1_000_000
PER_CALL = 20
WIDTH, HEIGHT = 3840, 2160


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device_index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "", 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "", 1).isdigit()]
        load = [v for v in sm if v > 500] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = []
        for k, nm in enumerate(names):
            if any(r[5 + k].lower() == "active" for r in self.rows):
                reasons.append(nm)
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def _reduce_device():
    """Where the rank reductions run: the GPU under NCCL, host memory under gloo."""
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def generate_cloud(seed, num_points=None, count=None):
    """Configuration 2's cloud for `seed` (num_points None: the configuration's
    100M). count: only its first `count` points -- a prefix of the same cloud,
    not a smaller cloud (the sensor path spans the configured size)."""
    from remobench_b200 import synth
    over = {"seed": seed}
    if num_points is not None:
        over["num_points"] = num_points
    cfg = synth.config(2, **over)
    t0 = time.time()
    pts = synth.generate(cfg, 0, count)
    bmin, bmax = synth.scene_box(cfg)
    return cfg, pts, bmin, bmax, time.time() - t0


def sample_identity(pts, sample_batches):
    """Which points a CPU sample covers: its first batch, count and a digest."""
    import hashlib
    n = min(len(pts), sample_batches * BATCH)
    h = hashlib.blake2b(np.ascontiguousarray(pts[:n]).view(np.uint8), digest_size=8).hexdigest()
    return {"first_batch": 0, "batches": sample_batches, "points": int(n), "blake2b_64": h}


def ncu_traffic(kernel):
    """The kernel's DRAM traffic per 1M-point launch from the committed ncu
    capture summary (profiles/ncu_traffic.json, written from an ncu capture of
    the build it names), or None with the reason when there is none or the
    kernel's source changed since the capture."""
    import hashlib
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            table = json.load(f)
    except Exception:
        return None, "no ncu capture summary"
    row = table.get("kernels", {}).get(kernel)
    if row is None:
        return None, f"no ncu capture of {kernel}"
    src = os.path.join(ROOT, row["source"])
    try:
        with open(src, "rb") as f:
            digest = hashlib.sha256(f.read()).hexdigest()[:16]
    except Exception:
        return None, f"{row['source']} missing"
    if digest != row["source_sha256_16"]:
        return None, f"{row['source']} changed since the capture ({row['captured']})"
    return row["dram_bytes_per_launch"], f"ncu capture {row['captured']}: {row['workload']}"


def cpu_baseline(pts, bmin, bmax, sample_batches, threads):
    """The oracle (CPU restatement of the reference's builder) on the first
    sample_batches batches of the same cloud: Update + Accumulate."""
    from oracle import binding as ob
    t = ob.Tree(num_threads=threads)
    t.reset(bmin, bmax)
    n = 0
    t0 = time.perf_counter()
    for b in range(sample_batches):
        chunk = pts[b * BATCH:(b + 1) * BATCH]
        t.add_batch(chunk)
        n += len(chunk)
        if (b + 1) % PER_CALL == 0 or b + 1 == sample_batches:
            t.accumulate(b + 1)
    dt = time.perf_counter() - t0
    t.close()
    return n / dt / 1e6, dt, n


def cpu_baseline_median(pts, bmin, bmax, sample_batches, threads, reps):
    """Median Mpts/s of `reps` runs of cpu_baseline, and the last run's time."""
    vals, dt = [], 0.0
    for _ in range(max(reps, 1)):
        v, dt, _ = cpu_baseline(pts, bmin, bmax, sample_batches, threads)
        vals.append(v)
    return statistics.median(vals), dt


def reference_kernels_b200(pts, bmin, bmax):
    """The reference's own kernels (kernels/remolod, NVRTC-compiled from its
    sources into oracle/_ref/ in the build container) timed on this GPU over
    the same cloud; None when they were not built or no GPU is visible."""
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_launcher.so")
    if not os.path.exists(lib):
        return {"unavailable": "oracle/_ref was not built (the reference sources are not mounted here)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
        from time_ref import time_kernels
        return time_kernels(pts, bmin, bmax, BATCH, "shipped")
    except Exception as e:  # reported, not fatal: the CPU arm stands on its own
        return {"unavailable": f"{type(e).__name__}: {e}"}


def run_reference(args, world, rank):
    """--impl reference: the reference path's CPU implementation (the oracle
    port; the reference's own code is GPU-only and GL-bound) on a bounded sample
    of the same workload -- the first cpu_sample_batches batches of the 100M
    cloud the repo arm ingests -- every host thread it can use. The reference's
    own GPU kernels, timed on the same box over the whole cloud, ride along as
    reference_kernels_b200 (not the line's value)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sample = args.cpu_sample_batches
    cfg, pts, bmin, bmax, _ = generate_cloud(1, count=sample * BATCH)
    for _ in range(args.warmup):
        cpu_baseline(pts, bmin, bmax, min(sample, 2), threads)
    value, dt = cpu_baseline_median(pts, bmin, bmax, sample, threads, args.steps)
    ident = sample_identity(pts, sample)
    kernels = None
    if not args.no_reference_kernels:
        del pts
        _, full, bmin, bmax, _ = generate_cloud(1)
        kernels = reference_kernels_b200(full, bmin, bmax)
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 points, int64 sums", "data": "synthetic",
            "config": {"workload": f"config 2 sample: first {sample} x 1M-point batches of the 100M-point "
                                   "2x2 km synthetic lidar cloud, Update+Accumulate",
                       "batch_points": BATCH, "sample": ident},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"first {sample} x 1M-point batches of the 100M-point cloud "
                                       f"(median of {args.steps} runs, {dt:.1f} s each), the restatement "
                                       f"on {threads} threads", "identity": ident},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_kernels_b200": kernels}
    print(json.dumps(line), flush=True)


def run_config5(args, world, rank, local):
    """The full streaming run (remobench_b200/streaming.py) on each rank's GPU;
    rank 0 prints its JSON line. Not the default step: it generates 16 GB of
    points and takes minutes."""
    import torch
    from remobench_b200 import streaming
    torch.cuda.set_device(local)
    clocks = ClockSampler(local)
    clocks.start()
    out = streaming.run(seed=1 + rank, log=lambda m: print(m, file=sys.stderr, flush=True))
    clk = clocks.stop()
    if rank == 0:
        line = {"metric": "config 5 streaming: ingest Mpts/s + frame ms at 7680x4320", "value": out["ingest_mpts_s"],
                "unit": "Mpts/s", "n_gpus": world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 points, int64/int128 sums", "data": "synthetic", "clocks": clk}
        line.update(out)
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--points", type=int, default=100_000_000)
    ap.add_argument("--frames", type=int, default=30)
    ap.add_argument("--cpu-sample-batches", type=int, default=20)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--config", type=int, default=2,
                    help="2: the benchmark (default); 5: the 1B-point full streaming run, its own JSON line")
    ap.add_argument("--no-reference-kernels", action="store_true",
                    help="reference arm: skip timing the reference's own GPU kernels")
    args = ap.parse_args()

    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        barrier(world)
        return
    if args.config == 5:
        run_config5(args, world, rank, local)
        barrier(world)
        return

    import ctypes

    import torch
    from remobench_b200 import capi
    from remobench_b200.camera import orbit_path
    from remobench_b200.lod import Context, make_frame

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg, pts, bmin, bmax, gen_s = generate_cloud(1 + rank, args.points if args.points != 100_000_000 else None)
    n = len(pts)
    nb = (n + BATCH - 1) // BATCH

    # the whole cloud resident in HBM as a ring of nb slots (batch b in slot b)
    host = torch.from_numpy(pts.view(np.float32).reshape(n, 4))
    pinned = host.pin_memory()
    ring = torch.zeros((nb, BATCH, 4), dtype=torch.float32, device=dev)
    ring.view(-1, 4)[:n].copy_(pinned, non_blocking=False)
    sizes = [min(BATCH, n - b * BATCH) for b in range(nb)]

    ctx = Context(device=local, ring_slots=nb, slot_capacity=BATCH, max_batches_per_build=PER_CALL,
                  time_budget_ms=0.0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.allocate(n, bmin, bmax)

    def ingest_resident():
        ctx.reset()
        consumed = 0
        while consumed < nb:
            r = ctx.build(ring, sizes, nb, nb)
            consumed = r.batches_consumed
            if r.batches_this_call == 0:
                raise RuntimeError("build made no progress")

    def ingest_host():
        ctx.reset()
        r = ctx.ingest_host(pinned, BATCH)
        if r.batches_consumed != nb:
            raise RuntimeError("host ingest stopped early")
        return ctx.stats()

    for _ in range(args.warmup):
        ingest_resident()
    torch.cuda.synchronize()
    def kernel_launches():
        # entries named k_* are launches; expand_pass counts passes inside k_expand_rest
        return sum(v["launches"] for k, v in ctx.profile().items() if k.startswith("k_"))

    launches0 = kernel_launches()

    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        ingest_resident()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_total = ev0.elapsed_time(ev1)
    launches = kernel_launches() - launches0
    ms_step = max_over_ranks(ms_total / args.steps, world)
    total_points = sum_over_ranks(float(n), world)
    value = total_points / (ms_step / 1e3) / 1e6

    # end to end from pinned host memory
    e2e = None
    if not args.no_e2e:
        ingest_host()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            st = ingest_host()
        e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
        e2e = {"value": round(total_points / (ems / 1e3) / 1e6, 3), "unit": UNIT,
               "h2d_bytes_per_step": int(n * 16), "d2h_bytes_per_step": int(ctypes.sizeof(capi.Stats)),
               "ms_per_step": round(ems, 3)}
        stats_e2e = st
    clk = clocks.stop()

    # the tree of the last resident ingest, then the raster along the orbit
    ingest_resident()
    stats = ctx.stats()
    fb = torch.empty(WIDTH * HEIGHT, dtype=torch.int64, device=dev)
    rgba = torch.empty(WIDTH * HEIGHT, dtype=torch.int32, device=dev)
    path = orbit_path(bmin, bmax, 300, seed=7)
    frame_ms, samples = [], []
    step = max(1, 300 // max(args.frames, 1))
    for k in range(0, 300, step):
        yaw, pitch, rs = path[k]
        f = make_frame(bmin, bmax, WIDTH, HEIGHT, yaw=yaw, pitch=pitch, radius_scale=rs, edl=True)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = ctx.render(f, fb, rgba)
        b.record(stream)
        torch.cuda.synchronize()
        frame_ms.append(a.elapsed_time(b))
        samples.append(r.draw_samples)
    frame_ms = frame_ms[1:] if len(frame_ms) > 1 else frame_ms

    # one profiled ingest: per-kernel CUDA-event durations for the roofline
    ctx.reset_profile()
    ctx.set_profiling(True)
    ingest_resident()
    ctx.set_profiling(False)
    prof = ctx.profile()
    upd = {k: v for k, v in prof.items() if v["timed"] > 0 and k not in ("k_reset_root",)}
    total_k = sum(v["ms"] for v in upd.values())
    top = max(upd.items(), key=lambda kv: kv[1]["ms"])
    # algorithmic bytes of a kernel per unit handed to it (points): the point
    # read (16 B), plus its leaf id (4 B) where one is written, plus the stored
    # point and index (20 B) for insertion
    bytes_per_unit = {"k_vox_sample": 16.0, "k_count_first": 20.0, "k_insert": 16.0 + 4.0 + 20.0,
                      "k_recount": 4.0, "k_accumulate": 16.0, "k_deep_bin": 4.0, "k_deep_move": 4.0}
    peak, peak_kind = peaks()
    roof = None
    if top[0] in bytes_per_unit and top[1]["units"] > 0:
        avg_ms = top[1]["ms"] / top[1]["timed"]
        per_launch_bytes = bytes_per_unit[top[0]] * top[1]["units"] / top[1]["launches"]
        achieved = per_launch_bytes / (avg_ms / 1e3) / 1e9
        traffic, traffic_note = ncu_traffic(top[0])
        roof = {"bound": "hbm", "kernel": top[0], "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 5), "peak_kind": peak_kind,
                "traffic": traffic, "traffic_unit": "DRAM bytes read + written per launch (ncu)",
                "traffic_source": traffic_note,
                "algorithmic_bytes_per_launch": round(per_launch_bytes),
                "avg_launch_ms": round(avg_ms, 4), "share": round(top[1]["ms"] / total_k, 3)}

    # the raster against the same HBM peak: per frame, clearing the packed
    # framebuffer (8 B/px), reading every drawn sample (16 B) and its 64-bit
    # atomicMin (8 B), EDL reading and writing each pixel (16 B/px) and the
    # resolve reading the packed and writing the RGBA pixel (12 B/px)
    raster_roof = None
    if frame_ms:
        p50_ms = float(np.percentile(frame_ms, 50))
        px = WIDTH * HEIGHT
        frame_bytes = px * (8 + 16 + 12) + float(np.median(samples)) * (16 + 8)
        ach = frame_bytes / (p50_ms / 1e3) / 1e9
        raster_roof = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                       "frac": round(ach / peak, 4), "peak_kind": peak_kind,
                       "algorithmic_bytes_per_frame": round(frame_bytes), "p50_ms": round(p50_ms, 4)}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_sample_batches > 0:
        threads = os.cpu_count() or 1
        v, dt = cpu_baseline_median(pts, bmin, bmax, args.cpu_sample_batches, threads, args.cpu_reps)
        cpu = {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"first {args.cpu_sample_batches} x 1M-point batches of the same cloud, "
                         f"Update+Accumulate, median of {args.cpu_reps} runs ({dt:.1f} s each) on "
                         f"{threads} threads",
               "identity": sample_identity(pts, args.cpu_sample_batches)}

    # the reference's own kernels over the same cloud on this GPU, beside the
    # line's value (not part of it)
    ref_kernels = None
    if rank == 0 and world == 1 and not args.no_reference_kernels:
        ref_kernels = reference_kernels_b200(pts, bmin, bmax)

    if rank == 0:
        p50 = float(np.percentile(frame_ms, 50)) if frame_ms else None
        p99 = float(np.percentile(frame_ms, 99)) if frame_ms else None
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 points, int64/int128 sums",
            "data": "synthetic",
            "config": {"workload": "config 2: 100M-point synthetic lidar cloud (2x2 km, 2000 boxes, 20000 poles), "
                                   "1M-point batches, 20 per build + Accumulate; raster 3840x2160 orbit",
                       "points": n, "batch_points": BATCH, "parallelism": f"replicas x{world}",
                       "l2": "inputs 1.6 GB > L2"},
            "raster_ms_per_frame": {"p50": round(p50, 3) if p50 else None, "p99": round(p99, 3) if p99 else None,
                                    "frames": len(frame_ms), "width": WIDTH, "height": HEIGHT,
                                    "mean_samples": int(np.mean(samples)) if samples else 0},
            "tree": {"nodes": stats.num_nodes, "voxels": stats.num_voxels, "points": stats.num_points,
                     "max_depth": stats.max_depth, "spilled": stats.spilled_points},
            "gpu_launches": int(launches),
            "roofline": roof,
            "raster_roofline": raster_roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "generate_s": round(gen_s, 1),
            "reference_kernels_b200": ref_kernels,
            "kernels": {k: {"launches": v["launches"] // 1, "ms": round(v["ms"], 3)} for k, v in
                        sorted(upd.items(), key=lambda kv: -kv[1]["ms"])},
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
