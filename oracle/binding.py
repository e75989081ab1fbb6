"""ctypes binding of the CPU oracle (oracle.c) -- test infrastructure only.

Loaded by tests/, the smoke entry point and the benchmark's CPU-baseline arm,
never by the product path. Builds liboracle.so on first use when it is missing
and a compiler is available.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


class Config(ctypes.Structure):
    _fields_ = [
        ("max_nodes", ctypes.c_uint32),
        ("max_points_per_node", ctypes.c_uint32),
        ("points_per_chunk", ctypes.c_uint32),
        ("max_expand_iters", ctypes.c_uint32),
        ("persistent_capacity", ctypes.c_uint64),
        ("safety_margin", ctypes.c_uint64),
        ("ring_slots", ctypes.c_uint32),
        ("slot_capacity", ctypes.c_uint32),
        ("max_batches_per_build", ctypes.c_uint32),
        ("num_threads", ctypes.c_uint32),
    ]


class NodeInfo(ctypes.Structure):
    _fields_ = [
        ("child", ctypes.c_int32 * 8),
        ("counter", ctypes.c_uint32),
        ("num_points", ctypes.c_uint32),
        ("level", ctypes.c_uint32),
        ("X", ctypes.c_uint32),
        ("Y", ctypes.c_uint32),
        ("Z", ctypes.c_uint32),
        ("grid", ctypes.c_int32),
        ("num_voxels", ctypes.c_uint32),
        ("num_point_chunks", ctypes.c_uint32),
        ("num_voxel_chunks", ctypes.c_uint32),
        ("is_leaf", ctypes.c_uint32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("num_nodes", ctypes.c_uint32),
        ("num_inner", ctypes.c_uint32),
        ("num_leaves", ctypes.c_uint32),
        ("num_nonempty_leaves", ctypes.c_uint32),
        ("num_points", ctypes.c_uint64),
        ("num_voxels", ctypes.c_uint64),
        ("num_chunks_points", ctypes.c_uint32),
        ("num_chunks_voxels", ctypes.c_uint32),
        ("batchlet_index", ctypes.c_uint32),
        ("num_points_processed", ctypes.c_uint64),
        ("num_allocated_chunks", ctypes.c_uint64),
        ("chunk_pool_size", ctypes.c_uint64),
        ("persistent_offset", ctypes.c_uint64),
        ("mem_capacity_reached", ctypes.c_uint32),
        ("node_pool_overflow", ctypes.c_uint32),
        ("max_points_per_node", ctypes.c_uint32),
        ("counter_underflows", ctypes.c_uint32),
        ("dropped_points", ctypes.c_uint64),
        ("expand_iters", ctypes.c_uint64),
        ("nodes_split", ctypes.c_uint64),
        ("spilled_points", ctypes.c_uint64),
        ("num_grids", ctypes.c_uint32),
        ("overflow_flags", ctypes.c_uint32),
    ]


class AccumI(ctypes.Structure):
    _fields_ = [
        ("s1", ctypes.c_uint64 * 3),
        ("s2_lo", ctypes.c_uint64 * 6),
        ("s2_hi", ctypes.c_uint64 * 6),
        ("c1", ctypes.c_uint64 * 3),
        ("c2", ctypes.c_uint64 * 3),
        ("count", ctypes.c_uint32),
        ("last_touched_batch", ctypes.c_uint32),
        ("state", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
    ]


class AccumF(ctypes.Structure):
    _fields_ = [
        ("g", ctypes.c_double * 9),
        ("c", ctypes.c_float * 6),
        ("count", ctypes.c_uint32),
        ("last_touched_batch", ctypes.c_uint32),
    ]


class AccumGlobals(ctypes.Structure):
    _fields_ = [
        ("morton_watermark", ctypes.c_uint64),
        ("num_accumulated", ctypes.c_uint64),
        ("sum_leaf_counts", ctypes.c_uint64),
        ("points_folded", ctypes.c_uint32),
        ("num_leaves_folded", ctypes.c_uint32),
        ("inner_with_sums", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
    ]


class AnalysisNode(ctypes.Structure):
    _fields_ = [
        ("eig", ctypes.c_double * 3),
        ("normal", ctypes.c_double * 3),
        ("surface_variation", ctypes.c_double),
        ("planarity", ctypes.c_double),
        ("count", ctypes.c_uint64),
    ]


class AnalysisParams(ctypes.Structure):
    _fields_ = [("min_points", ctypes.c_uint32), ("closure_margin", ctypes.c_uint32),
                ("current_batch", ctypes.c_uint32), ("frontier_only", ctypes.c_uint32),
                ("pixel_budget", ctypes.c_float), ("pad", ctypes.c_uint32)]


class Frame(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_float),
        ("height", ctypes.c_float),
        ("transform", ctypes.c_float * 16),
        ("transform_frozen", ctypes.c_float * 16),
        ("box_min", ctypes.c_float * 3),
        ("box_max", ctypes.c_float * 3),
        ("lod_pixel_budget", ctypes.c_float),
        ("point_size", ctypes.c_int32),
        ("drawlist_capacity", ctypes.c_uint32),
        ("force_large", ctypes.c_void_p),
        ("color_mode", ctypes.c_int32),
    ]


class RenderResult(ctypes.Structure):
    _fields_ = [
        ("draw_items", ctypes.c_uint32),
        ("drawlist_overflow", ctypes.c_uint32),
        ("draw_samples", ctypes.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        L.or_create.restype = vp
        L.or_create.argtypes = [ctypes.POINTER(Config)]
        L.or_destroy.argtypes = [vp]
        L.or_reset.argtypes = [vp, ctypes.POINTER(ctypes.c_float * 3), ctypes.POINTER(ctypes.c_float * 3)]
        L.or_add_batch.argtypes = [vp, vp, u32]
        L.or_add_batch.restype = ctypes.c_int
        L.or_build.argtypes = [vp, vp, vp, u32]
        L.or_build.restype = u32
        L.or_sweep.argtypes = [vp]
        L.or_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        L.or_num_nodes.argtypes = [vp]
        L.or_num_nodes.restype = u32
        L.or_get_node.argtypes = [vp, u32, ctypes.POINTER(NodeInfo)]
        L.or_leaf_points.argtypes = [vp, u32, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.or_leaf_points.restype = u32
        L.or_node_voxels.argtypes = [vp, u32, ctypes.POINTER(vp)]
        L.or_node_voxels.restype = u32
        L.or_node_grid.argtypes = [vp, u32]
        L.or_node_grid.restype = vp
        L.or_accumulate.argtypes = [vp, u32, ctypes.POINTER(AccumGlobals)]
        L.or_get_accum_i.argtypes = [vp, u32, ctypes.POINTER(AccumI)]
        L.or_get_accum_f.argtypes = [vp, u32, ctypes.POINTER(AccumF)]
        L.or_analyze_fp64.argtypes = [vp, vp]
        L.or_sym3_eig_jacobi.argtypes = [vp, vp, vp]
        L.or_render.argtypes = [vp, ctypes.POINTER(Frame), vp, ctypes.POINTER(RenderResult), vp]
        L.or_rolled_sums.argtypes = [vp, vp, vp]
        L.or_analysis_scores.argtypes = [vp, ctypes.POINTER(Frame), ctypes.POINTER(AnalysisParams), vp, vp, vp, vp, vp]
        L.or_render_flat.argtypes = [vp, u64, ctypes.POINTER(Frame), vp]
        L.or_edl.argtypes = [vp, u32, u32, ctypes.c_float]
        L.or_wireframe.argtypes = [vp, ctypes.POINTER(Frame), vp, vp, u32]
        L.or_features.argtypes = [vp, u32, u32, vp]
        L.or_refine_colors.argtypes = [vp, vp, u32, u32, ctypes.POINTER(u32), ctypes.POINTER(u64)]
        L.or_deepen.argtypes = [vp, vp, u32, u32, ctypes.POINTER(u32)]
        L.or_collapse.argtypes = [vp, vp, u32, u32, ctypes.POINTER(u32), ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.or_deepen.restype = ctypes.c_int
        _lib = L
    return _lib


POINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("color", "<u4")])


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Tree:
    """The oracle's octree: reset, add batches, read nodes back."""

    def __init__(self, **cfg):
        c = Config()
        for k, v in cfg.items():
            setattr(c, k, v)
        self._cfg = c
        self.h = lib().or_create(ctypes.byref(c))
        if not self.h:
            raise MemoryError("or_create failed")

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def reset(self, box_min, box_max):
        bmin = (ctypes.c_float * 3)(*box_min)
        bmax = (ctypes.c_float * 3)(*box_max)
        lib().or_reset(self.h, ctypes.byref(bmin), ctypes.byref(bmax))

    def add_batch(self, pts):
        pts = np.ascontiguousarray(pts)
        return lib().or_add_batch(self.h, _ptr(pts), len(pts))

    def build(self, ring, batch_sizes, num_uploaded):
        ring = np.ascontiguousarray(ring)
        bs = np.ascontiguousarray(batch_sizes, dtype=np.uint32)
        return lib().or_build(self.h, _ptr(ring), _ptr(bs), num_uploaded)

    def sweep(self):
        lib().or_sweep(self.h)

    def stats(self):
        s = Stats()
        lib().or_get_stats(self.h, ctypes.byref(s))
        return s

    def num_nodes(self):
        return lib().or_num_nodes(self.h)

    def node(self, i):
        n = NodeInfo()
        if lib().or_get_node(self.h, i, ctypes.byref(n)) != 0:
            raise IndexError(i)
        return n

    def node_table(self):
        """Structured array of every node."""
        nn = self.num_nodes()
        dt = np.dtype([("child", "<i4", 8), ("counter", "<u4"), ("num_points", "<u4"),
                       ("level", "<u4"), ("X", "<u4"), ("Y", "<u4"), ("Z", "<u4"),
                       ("grid", "<i4"), ("num_voxels", "<u4"), ("num_point_chunks", "<u4"),
                       ("num_voxel_chunks", "<u4"), ("is_leaf", "<u4")])
        out = np.zeros(nn, dtype=dt)
        buf = np.zeros(1, dtype=dt)
        for i in range(nn):
            n = self.node(i)
            ctypes.memmove(buf.ctypes.data, ctypes.addressof(n), dt.itemsize)
            out[i] = buf[0]
        return out

    def leaf_points(self, i):
        p, ix = ctypes.c_void_p(), ctypes.c_void_p()
        n = lib().or_leaf_points(self.h, i, ctypes.byref(p), ctypes.byref(ix))
        if n == 0:
            return np.zeros(0, POINT_DTYPE), np.zeros(0, np.uint32)
        pts = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), (n * 16,))
        idx = np.ctypeslib.as_array(ctypes.cast(ix, ctypes.POINTER(ctypes.c_uint32)), (n,))
        return pts.view(POINT_DTYPE).copy(), idx.copy()

    def node_voxels(self, i):
        p = ctypes.c_void_p()
        n = lib().or_node_voxels(self.h, i, ctypes.byref(p))
        if n == 0:
            return np.zeros(0, POINT_DTYPE)
        v = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), (n * 16,))
        return v.view(POINT_DTYPE).copy()

    def node_grid(self, i):
        p = lib().or_node_grid(self.h, i)
        if not p:
            return None
        g = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint32)), (65536,))
        return g.copy()

    def features(self, current_batch, closure_margin):
        """(num_nodes, 16) float32: the learned scorer's inputs per node."""
        out = np.zeros((self.num_nodes(), 16), dtype=np.float32)
        lib().or_features(self.h, current_batch, closure_margin, _ptr(out))
        return out

    def refine_colors(self, nodes, capacity=2097152):
        """Colour filtering of the nodes' voxels; (nodes filtered, voxels filtered)."""
        arr = np.ascontiguousarray(nodes, dtype=np.uint32)
        m, v = ctypes.c_uint32(), ctypes.c_uint64()
        lib().or_refine_colors(self.h, _ptr(arr), len(arr), capacity, ctypes.byref(m), ctypes.byref(v))
        return m.value, v.value

    def deepen(self, nodes, min_points=0):
        """Refinement's deepening of the leaves among `nodes`; (refused by the
        memory check, leaves taken)."""
        arr = np.ascontiguousarray(nodes, dtype=np.uint32)
        m = ctypes.c_uint32()
        rc = lib().or_deepen(self.h, _ptr(arr), len(arr), min_points, ctypes.byref(m))
        return rc != 0, m.value

    def collapse(self, nodes, max_points=0):
        """Refinement's collapsing of the listed nodes; (collapsed, points moved,
        voxels dropped)."""
        arr = np.ascontiguousarray(nodes, dtype=np.uint32)
        m, p, v = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
        lib().or_collapse(self.h, _ptr(arr), len(arr), max_points, ctypes.byref(m), ctypes.byref(p), ctypes.byref(v))
        return m.value, p.value, v.value

    def accumulate(self, batch_index):
        g = AccumGlobals()
        lib().or_accumulate(self.h, batch_index, ctypes.byref(g))
        return g

    def accum_i(self, i):
        a = AccumI()
        lib().or_get_accum_i(self.h, i, ctypes.byref(a))
        return a

    def accum_f(self, i):
        a = AccumF()
        lib().or_get_accum_f(self.h, i, ctypes.byref(a))
        return a

    def analyze_fp64(self):
        nn = self.num_nodes()
        arr = (AnalysisNode * max(nn, 1))()
        lib().or_analyze_fp64(self.h, ctypes.cast(arr, ctypes.c_void_p))
        return arr

    def rolled_sums(self):
        nn = self.num_nodes()
        out = np.zeros((nn, 16), dtype=np.uint64)
        lt = np.zeros(nn, dtype=np.uint32)
        lib().or_rolled_sums(self.h, _ptr(out), _ptr(lt))
        return out, lt

    def analysis_scores(self, frame, params, analysis):
        nn = self.num_nodes()
        cov = np.zeros(nn, dtype=np.float32)
        flags = np.zeros(nn, dtype=np.uint32)
        closed = np.zeros(nn, dtype=np.uint32)
        score = np.zeros(nn, dtype=np.float64)
        lib().or_analysis_scores(self.h, ctypes.byref(frame), ctypes.byref(params), ctypes.cast(analysis, ctypes.c_void_p),
                                 _ptr(cov), _ptr(flags), _ptr(closed), _ptr(score))
        return cov, flags, closed, score

    def render(self, frame, item_nodes_cap=0):
        w, h = int(frame.width), int(frame.height)
        fb = np.zeros(w * h, dtype=np.uint64)
        r = RenderResult()
        items = None
        if item_nodes_cap:
            items = np.zeros(item_nodes_cap, dtype=np.uint32)
        lib().or_render(self.h, ctypes.byref(frame), _ptr(fb), ctypes.byref(r),
                        _ptr(items) if items is not None else None)
        return fb, r, items


def wireframe(tree, frame, fb, item_nodes):
    """The draw items' box edges drawn into fb (a copy is returned)."""
    out = np.array(fb, dtype=np.uint64, copy=True)
    items = np.ascontiguousarray(item_nodes, dtype=np.uint32)
    lib().or_wireframe(tree.h, ctypes.byref(frame), _ptr(out), _ptr(items), len(items))
    return out


def render_flat(points, frame):
    w, h = int(frame.width), int(frame.height)
    fb = np.zeros(w * h, dtype=np.uint64)
    pts = np.ascontiguousarray(points)
    lib().or_render_flat(_ptr(pts), len(pts), ctypes.byref(frame), _ptr(fb))
    return fb


def edl(fb, width, height, strength):
    out = np.array(fb, dtype=np.uint64, copy=True)
    lib().or_edl(_ptr(out), width, height, strength)
    return out


def sym3_eig(a6):
    a = np.ascontiguousarray(a6, dtype=np.float64)
    e = np.zeros(3)
    v = np.zeros(3)
    lib().or_sym3_eig_jacobi(_ptr(a), _ptr(e), _ptr(v))
    return e, v
