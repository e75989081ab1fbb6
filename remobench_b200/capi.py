"""ctypes binding of the C ABI (include/rb_capi.h) exported by lib/librb_cuda.so.

This is the Python face of the drop-in boundary: the same entry points the
C++ host (ILodPipeline implementations) calls. No torch types cross it;
device buffers are passed as integer addresses.
"""
import ctypes
import os

_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "librb_cuda.so")

RB_OK = 0
STATUS_NAMES = {0: "RB_OK", 1: "RB_ERR_INVALID_ARG", 2: "RB_ERR_CUDA", 3: "RB_ERR_OUT_OF_MEMORY",
                4: "RB_ERR_STATE", 5: "RB_ERR_RING", 6: "RB_ERR_CAPACITY", 7: "RB_ERR_NO_DEVICE",
                8: "RB_ERR_UNSUPPORTED"}
RB_ERR_INVALID_ARG, RB_ERR_CUDA, RB_ERR_OUT_OF_MEMORY, RB_ERR_STATE = 1, 2, 3, 4
RB_ERR_RING, RB_ERR_CAPACITY, RB_ERR_NO_DEVICE, RB_ERR_UNSUPPORTED = 5, 6, 7, 8
RB_PIPELINE_REMOLOD, RB_PIPELINE_SIMLOD, RB_PIPELINE_FLAT = 0, 1, 2
RB_VOXEL_LOWEST_INDEX, RB_VOXEL_FIRST_COME = 0, 1
RB_SCORE_PARTIAL, RB_SCORE_CLOSED, RB_SCORE_LEARNED = 0, 1, 2
RB_COLOR_RGB, RB_COLOR_BY_NODE, RB_COLOR_BY_LOD, RB_COLOR_WHITE = 0, 1, 2, 3
MLP_NUM_PARAMS, NUM_FEATURES = 5378, 16

u32, u64, i32, f32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_float


class Config(ctypes.Structure):
    _fields_ = [("struct_size", u32), ("pipeline", u32), ("device", i32), ("max_nodes", u32),
                ("max_points_per_node", u32), ("points_per_chunk", u32), ("max_expand_iters", u32),
                ("ring_slots", u32), ("slot_capacity", u32), ("max_batches_per_build", u32),
                ("time_budget_ms", f32), ("voxel_mode", u32), ("accumulate", u32),
                ("spilled_capacity", u32), ("spilling_nodes_capacity", u32), ("drawlist_capacity", u32),
                ("safety_margin", u64), ("use_graphs", u32), ("backlog_capacity", u32),
                ("store_capacity", u64), ("refine_voxel_capacity", u32), ("reserved", u32 * 3)]


class CloudMeta(ctypes.Structure):
    _fields_ = [("num_points", u64), ("box_min", f32 * 3), ("box_max", f32 * 3)]


class BatchView(ctypes.Structure):
    _fields_ = [("slots", u64), ("batch_sizes", ctypes.POINTER(u32)), ("num_batches_uploaded", u32),
                ("slot_capacity", u32), ("num_slots", u32), ("num_batches_total", u32)]


class Frame(ctypes.Structure):
    _fields_ = [("width", f32), ("height", f32), ("transform", f32 * 16), ("transform_frozen", f32 * 16),
                ("box_min", f32 * 3), ("box_max", f32 * 3), ("lod_pixel_budget", f32), ("point_size", i32),
                ("enable_edl", u32), ("edl_strength", f32), ("frame_counter", u64), ("color_mode", i32),
                ("show_bounding_box", u32)]


class BuildResult(ctypes.Structure):
    _fields_ = [("batches_consumed", u32), ("batches_this_call", u32), ("more", u32),
                ("mem_capacity_reached", u32), ("device_ms", f32), ("pad", u32)]


class Stats(ctypes.Structure):
    _fields_ = [("num_points", u64), ("num_voxels", u64), ("num_points_ingested", u64), ("num_nodes", u32),
                ("num_inner", u32), ("num_leaves", u32), ("num_nonempty_leaves", u32), ("max_depth", u32),
                ("max_points_per_node", u32), ("num_chunks_points", u32), ("num_chunks_voxels", u32),
                ("batchlet_index", u32), ("counter_underflows", u32), ("num_allocated_chunks", u64),
                ("chunk_pool_size", u64), ("persistent_offset", u64), ("persistent_capacity", u64),
                ("bytes_allocated", u64), ("dropped_points", u64), ("expand_iters", u64),
                ("nodes_split", u64), ("spilled_points", u64), ("num_grids", u32), ("overflow_flags", u32),
                ("mem_capacity_reached", u32), ("node_capacity_reached", u32), ("num_visible_nodes", u32),
                ("pad", u32), ("num_visible_samples", u64)]


class RefineResult(ctypes.Structure):
    _fields_ = [("nodes_filtered", u32), ("voxels_filtered", u32), ("points_visited", u64)]


class DeepenResult(ctypes.Structure):
    _fields_ = [("nodes_selected", u32), ("nodes_split", u32), ("nodes_refused", u32), ("stopped", u32),
                ("points_moved", u64), ("voxels_made", u64)]


class CollapseResult(ctypes.Structure):
    _fields_ = [("nodes_collapsed", u32), ("grids_returned", u32), ("points_moved", u64), ("voxels_dropped", u64)]


class RenderResult(ctypes.Structure):
    _fields_ = [("draw_items", u32), ("drawlist_overflow", u32), ("draw_samples", u64), ("device_ms", f32),
                ("pad", u32)]


class AccumGlobals(ctypes.Structure):
    _fields_ = [("morton_watermark", u64), ("num_accumulated", u64), ("sum_leaf_counts", u64),
                ("points_folded", u32), ("num_leaves_folded", u32), ("inner_with_sums", u32), ("pad", u32)]


class Accum(ctypes.Structure):
    _fields_ = [("s1", u64 * 3), ("s2_lo", u64 * 6), ("s2_hi", u64 * 6), ("c1", u64 * 3), ("c2", u64 * 3),
                ("count", u32), ("last_touched_batch", u32), ("state", u32), ("pad", u32)]


class NodeInfo(ctypes.Structure):
    _fields_ = [("child", i32 * 8), ("counter", u32), ("num_points", u32), ("level", u32), ("X", u32),
                ("Y", u32), ("Z", u32), ("has_grid", u32), ("num_voxels", u32), ("num_point_chunks", u32),
                ("num_voxel_chunks", u32), ("is_leaf", u32)]


class AnalysisParams(ctypes.Structure):
    _fields_ = [("min_points", u32), ("closure_margin", u32), ("frontier_only", u32), ("queue_capacity", u32),
                ("pixel_budget", f32), ("score_mode", u32)]


class AnalysisResult(ctypes.Structure):
    _fields_ = [("queue_length", u32), ("eligible", u32), ("fp64_branch", u32), ("overflow", u32),
                ("device_ms", f32), ("pad", u32)]


class NodeAnalysis(ctypes.Structure):
    _fields_ = [("eig", f32 * 3), ("normal", f32 * 3), ("surface_variation", f32), ("planarity", f32),
                ("coverage", f32), ("score", f32), ("count", u64), ("last_touched", u32), ("closed", u32),
                ("flags", u32), ("pad", u32)]


class KernelProfile(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", u64), ("timed_launches", u64),
                ("total_ms", ctypes.c_double), ("units", u64)]


# name -> (restype, argtypes); the declarations of include/rb_capi.h
_vp = ctypes.c_void_p
SIGNATURES = {
    "rb_abi_version": (u32, []),
    "rb_status_string": (ctypes.c_char_p, [i32]),
    "rb_config_defaults": (None, [ctypes.POINTER(Config)]),
    "rb_create": (i32, [ctypes.POINTER(Config), ctypes.POINTER(_vp)]),
    "rb_destroy": (None, [_vp]),
    "rb_last_error": (ctypes.c_char_p, [_vp]),
    "rb_set_stream": (i32, [_vp, _vp]),
    "rb_allocate": (i32, [_vp, ctypes.POINTER(CloudMeta), u64]),
    "rb_release": (None, [_vp]),
    "rb_reset": (i32, [_vp]),
    "rb_build": (i32, [_vp, ctypes.POINTER(BatchView), ctypes.POINTER(BuildResult)]),
    "rb_ingest_host": (i32, [_vp, _vp, u64, u32, ctypes.POINTER(BuildResult)]),
    "rb_accumulate": (i32, [_vp, u32, ctypes.POINTER(AccumGlobals)]),
    "rb_render": (i32, [_vp, ctypes.POINTER(Frame), u64, u64, u64, ctypes.POINTER(RenderResult)]),
    "rb_render_noalloc": (i32, [_vp, ctypes.POINTER(Frame), u64, u64, u64, ctypes.POINTER(RenderResult)]),
    "rb_render_flat": (i32, [_vp, ctypes.POINTER(Frame), u64, u64, u64, u64, ctypes.POINTER(RenderResult)]),
    "rb_read_stats": (i32, [_vp, ctypes.POINTER(Stats)]),
    "rb_read_nodes": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_read_node_points": (i32, [_vp, u32, _vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_read_node_voxels": (i32, [_vp, u32, _vp, u32, ctypes.POINTER(u32)]),
    "rb_read_node_grid": (i32, [_vp, u32, _vp]),
    "rb_read_accums": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_analyze": (i32, [_vp, ctypes.POINTER(Frame), ctypes.POINTER(AnalysisParams), ctypes.POINTER(AnalysisResult)]),
    "rb_read_analysis": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_read_queue": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_read_rollup": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_refine": (i32, [_vp, u32, u64]),
    "rb_refine_colors": (i32, [_vp, u32, ctypes.POINTER(RefineResult)]),
    "rb_refine_deepen": (i32, [_vp, u32, u32, ctypes.POINTER(DeepenResult)]),
    "rb_refine_collapse": (i32, [_vp, _vp, u32, u32, ctypes.POINTER(CollapseResult)]),
    "rb_read_features": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_mlp_init": (i32, [_vp, u64]),
    "rb_mlp_set_params": (i32, [_vp, _vp]),
    "rb_mlp_get_params": (i32, [_vp, _vp]),
    "rb_mlp_predict": (i32, [_vp, u64, u32, u64]),
    "rb_mlp_gradients": (i32, [_vp, u64, u64, u32, _vp, ctypes.POINTER(f32)]),
    "rb_mlp_train_step": (i32, [_vp, u64, u64, u32, f32, ctypes.POINTER(f32)]),
    "rb_set_profiling": (i32, [_vp, ctypes.c_int]),
    "rb_read_profile": (i32, [_vp, _vp, u32, ctypes.POINTER(u32)]),
    "rb_reset_profile": (i32, [_vp]),
}

_lib = None


def lib():
    """The loaded librb_cuda.so with typed entry points. Raises if it is missing:
    there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise RuntimeError(f"{_LIB} is missing; build it with `python -m remobench_b200.build`")
        L = ctypes.CDLL(_LIB)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class RBError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def default_config(**overrides):
    c = Config()
    lib().rb_config_defaults(ctypes.byref(c))
    for k, v in overrides.items():
        setattr(c, k, v)
    return c
