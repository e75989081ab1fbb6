"""The C ABI library loads, exports every entry point include/rb_capi.h
declares, and its structs have the layout the ctypes binding assumes."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from remobench_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rb_capi.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rb_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = capi.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    assert set(names) == set(capi.SIGNATURES)


def test_abi_version_and_status_strings():
    lib = capi.lib()
    assert lib.rb_abi_version() == 2
    assert lib.rb_status_string(0) == b"ok"
    assert lib.rb_status_string(5) == b"ring depth mismatch"


STRUCTS = ["rb_kernel_profile", "rb_config", "rb_cloud_meta", "rb_batch_view", "rb_frame", "rb_build_result", "rb_stats",
           "rb_render_result", "rb_accum_globals", "rb_accum", "rb_node_info", "rb_point",
           "rb_deepen_result", "rb_collapse_result", "rb_refine_result"]
PY = {"rb_kernel_profile": capi.KernelProfile, "rb_config": capi.Config, "rb_cloud_meta": capi.CloudMeta, "rb_batch_view": capi.BatchView,
      "rb_frame": capi.Frame, "rb_build_result": capi.BuildResult, "rb_stats": capi.Stats,
      "rb_render_result": capi.RenderResult, "rb_accum_globals": capi.AccumGlobals, "rb_accum": capi.Accum,
      "rb_node_info": capi.NodeInfo, "rb_deepen_result": capi.DeepenResult,
      "rb_collapse_result": capi.CollapseResult, "rb_refine_result": capi.RefineResult}


def test_struct_layouts_match_header():
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"rb_capi.h\"\nint main(void){\n"
    for s in STRUCTS:
        src += f'printf("{s} %zu\\n", sizeof({s}));\n'
    src += 'printf("stats.num_visible_samples %zu\\n", offsetof(rb_stats, num_visible_samples));\n'
    src += 'printf("frame.frame_counter %zu\\n", offsetof(rb_frame, frame_counter));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write(src)
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        out = subprocess.check_output([exe]).decode().split("\n")
    sizes = dict(line.split() for line in out if line.strip())
    for s, cls in PY.items():
        assert int(sizes[s]) == ctypes.sizeof(cls), s
    assert int(sizes["rb_point"]) == 16
    assert int(sizes["stats.num_visible_samples"]) == capi.Stats.num_visible_samples.offset
    assert int(sizes["frame.frame_counter"]) == capi.Frame.frame_counter.offset


def test_config_defaults_are_the_reference_constants():
    c = capi.default_config()
    # kernels/remolod/remolod_structures.cuh:12-25, remolod_octree.cu:26-76, remolod_render.cu:22
    assert (c.max_nodes, c.max_points_per_node, c.points_per_chunk) == (200000, 50000, 1000)
    assert (c.ring_slots, c.slot_capacity, c.max_batches_per_build) == (50, 1000000, 20)
    assert (c.spilled_capacity, c.spilling_nodes_capacity, c.drawlist_capacity) == (10000000, 100000, 131072)
    assert c.safety_margin == 200000000 and c.max_expand_iters == 20


def test_create_validates_and_fails_loudly_without_gpu():
    lib = capi.lib()
    c = capi.default_config()
    h = ctypes.c_void_p()
    bad = capi.default_config(struct_size=4)
    assert lib.rb_create(ctypes.byref(bad), ctypes.byref(h)) == capi.RB_ERR_INVALID_ARG
    # the cell table takes 2 x backlog_capacity 16-byte slots: 2^28 (8 GB) is the limit
    bad = capi.default_config(backlog_capacity=(1 << 28) + 1)
    assert lib.rb_create(ctypes.byref(bad), ctypes.byref(h)) == capi.RB_ERR_INVALID_ARG
    assert c.backlog_capacity == 0  # 0: sized from slot_capacity
    st = lib.rb_create(ctypes.byref(c), ctypes.byref(h))
    import torch
    if torch.cuda.is_available():
        assert st == capi.RB_OK
        lib.rb_destroy(h)
    else:
        assert st == capi.RB_ERR_NO_DEVICE


def test_product_path_has_no_cpu_fallback():
    # the package never imports, links or loads the oracle
    pkg = os.path.join(ROOT, "remobench_b200")
    pat = re.compile(r"(import\s+oracle|from\s+oracle|liboracle|oracle\.binding|oracle/)")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cpp", ".cu", ".h", ".c")):
                text = open(os.path.join(dirpath, f), errors="replace").read()
                assert not pat.search(text), f


def test_refinement_calls_reject_a_missing_context():
    lib = capi.lib()
    d, r = capi.DeepenResult(), capi.CollapseResult()
    ids = (ctypes.c_uint32 * 2)(1, 2)
    assert lib.rb_refine_deepen(None, 8, 0, ctypes.byref(d)) == capi.RB_ERR_INVALID_ARG
    assert lib.rb_refine_collapse(None, ids, 2, 0, ctypes.byref(r)) == capi.RB_ERR_INVALID_ARG
