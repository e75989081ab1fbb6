"""Python face of the C ABI: a context object over lib/librb_cuda.so.

Device memory comes from torch (plumbing only); every stage runs in the CUDA
library. Nothing here computes LOD results on the CPU: if the library or a
GPU is missing, construction raises.
"""
import ctypes

import numpy as np

from . import capi
from .camera import frame_matrices

POINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("color", "<u4")])
NODE_DTYPE = np.dtype([("child", "<i4", 8), ("counter", "<u4"), ("num_points", "<u4"), ("level", "<u4"),
                       ("X", "<u4"), ("Y", "<u4"), ("Z", "<u4"), ("has_grid", "<u4"), ("num_voxels", "<u4"),
                       ("num_point_chunks", "<u4"), ("num_voxel_chunks", "<u4"), ("is_leaf", "<u4")])
ANALYSIS_DTYPE = np.dtype([("eig", "<f4", 3), ("normal", "<f4", 3), ("surface_variation", "<f4"),
                           ("planarity", "<f4"), ("coverage", "<f4"), ("score", "<f4"), ("count", "<u8"),
                           ("last_touched", "<u4"), ("closed", "<u4"), ("flags", "<u4"), ("pad", "<u4")])
ACCUM_DTYPE = np.dtype([("s1", "<u8", 3), ("s2_lo", "<u8", 6), ("s2_hi", "<u8", 6), ("c1", "<u8", 3),
                        ("c2", "<u8", 3), ("count", "<u4"), ("last_touched_batch", "<u4"), ("state", "<u4"),
                        ("pad", "<u4")])


def _check(ctx_handle, status):
    if status != capi.RB_OK:
        msg = capi.lib().rb_last_error(ctx_handle) if ctx_handle else b""
        raise capi.RBError(status, (msg or b"").decode(errors="replace"))


def make_frame(box_min, box_max, width, height, transform=None, frozen=None, budget=128.0, point_size=1,
               edl=False, edl_strength=0.4, **orbit):
    f = capi.Frame()
    f.width = float(width)
    f.height = float(height)
    if transform is None:
        transform = frame_matrices(box_min, box_max, width, height, **orbit)
    if frozen is None:
        frozen = transform
    for i, v in enumerate(np.asarray(transform, dtype=np.float32).reshape(-1)):
        f.transform[i] = float(v)
    for i, v in enumerate(np.asarray(frozen, dtype=np.float32).reshape(-1)):
        f.transform_frozen[i] = float(v)
    for a in range(3):
        f.box_min[a] = float(box_min[a])
        f.box_max[a] = float(box_max[a])
    f.lod_pixel_budget = float(budget)
    f.point_size = int(point_size)
    f.enable_edl = 1 if edl else 0
    f.edl_strength = float(edl_strength)
    return f


class Context:
    """One LOD pipeline instance (remolod / simlod / flat) behind the C ABI."""

    def __init__(self, **config):
        import torch
        self.torch = torch
        if not torch.cuda.is_available():
            raise capi.RBError(capi.RB_ERR_NO_DEVICE, "CUDA is not available")
        self.cfg = capi.default_config(**config)
        h = ctypes.c_void_p()
        st = capi.lib().rb_create(ctypes.byref(self.cfg), ctypes.byref(h))
        _check(None, st)
        self.h = h
        self.box_min = None
        self.box_max = None

    def close(self):
        h = getattr(self, "h", None)
        if not h:
            return
        self.h = None
        # at interpreter exit the module's globals may already be gone; the
        # process ending releases the context then
        lib = getattr(capi, "lib", None)
        if callable(lib):
            lib().rb_destroy(h)

    def __del__(self):
        self.close()

    def _ok(self, st):
        _check(self.h, st)

    def allocate(self, num_points, box_min, box_max, budget_bytes=0):
        m = capi.CloudMeta()
        m.num_points = int(num_points)
        for a in range(3):
            m.box_min[a] = float(box_min[a])
            m.box_max[a] = float(box_max[a])
        self.box_min = np.asarray(box_min, dtype=np.float32)
        self.box_max = np.asarray(box_max, dtype=np.float32)
        self._ok(capi.lib().rb_allocate(self.h, ctypes.byref(m), int(budget_bytes)))

    def reset(self):
        self._ok(capi.lib().rb_reset(self.h))

    def build(self, ring_tensor, batch_sizes, num_uploaded, num_total):
        """rb_build over a device ring tensor shaped (slots, slot_capacity, 4) float32."""
        sizes = (ctypes.c_uint32 * len(batch_sizes))(*[int(b) for b in batch_sizes])
        v = capi.BatchView()
        v.slots = ring_tensor.data_ptr()
        v.batch_sizes = sizes
        v.num_batches_uploaded = int(num_uploaded)
        v.slot_capacity = int(ring_tensor.shape[1])
        v.num_slots = int(ring_tensor.shape[0])
        v.num_batches_total = int(num_total)
        r = capi.BuildResult()
        self._ok(capi.lib().rb_build(self.h, ctypes.byref(v), ctypes.byref(r)))
        return r

    def ingest_host(self, points, batch_size):
        """rb_ingest_host from a host array (numpy POINT_DTYPE or a pinned torch tensor)."""
        if hasattr(points, "data_ptr"):
            ptr, n = points.data_ptr(), points.shape[0]
        else:
            ptr, n = points.ctypes.data, len(points)
        r = capi.BuildResult()
        self._ok(capi.lib().rb_ingest_host(self.h, ctypes.c_void_p(ptr), int(n), int(batch_size),
                                           ctypes.byref(r)))
        return r

    def accumulate(self, batch_index):
        g = capi.AccumGlobals()
        self._ok(capi.lib().rb_accumulate(self.h, int(batch_index), ctypes.byref(g)))
        return g

    def render(self, frame, fb, rgba=None, force_large=None):
        r = capi.RenderResult()
        self._ok(capi.lib().rb_render(self.h, ctypes.byref(frame), fb.data_ptr(),
                                      rgba.data_ptr() if rgba is not None else 0,
                                      force_large.data_ptr() if force_large is not None else 0,
                                      ctypes.byref(r)))
        return r

    def render_flat(self, frame, points_dev, fb, rgba=None):
        r = capi.RenderResult()
        self._ok(capi.lib().rb_render_flat(self.h, ctypes.byref(frame), points_dev.data_ptr(),
                                           int(points_dev.shape[0]), fb.data_ptr(),
                                           rgba.data_ptr() if rgba is not None else 0, ctypes.byref(r)))
        return r

    def stats(self):
        s = capi.Stats()
        self._ok(capi.lib().rb_read_stats(self.h, ctypes.byref(s)))
        return s

    def nodes(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_nodes(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=NODE_DTYPE)
        self._ok(capi.lib().rb_read_nodes(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n)))
        return out

    def node_points(self, i):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_node_points(self.h, i, None, None, 0, ctypes.byref(n)))
        pts = np.zeros(n.value, dtype=POINT_DTYPE)
        idx = np.zeros(n.value, dtype=np.uint32)
        if n.value:
            self._ok(capi.lib().rb_read_node_points(self.h, i, ctypes.c_void_p(pts.ctypes.data),
                                                    ctypes.c_void_p(idx.ctypes.data), n.value, ctypes.byref(n)))
        return pts, idx

    def node_voxels(self, i):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_node_voxels(self.h, i, None, 0, ctypes.byref(n)))
        v = np.zeros(n.value, dtype=POINT_DTYPE)
        if n.value:
            self._ok(capi.lib().rb_read_node_voxels(self.h, i, ctypes.c_void_p(v.ctypes.data), n.value,
                                                    ctypes.byref(n)))
        return v

    def node_grid(self, i):
        g = np.zeros(65536, dtype=np.uint32)
        self._ok(capi.lib().rb_read_node_grid(self.h, i, ctypes.c_void_p(g.ctypes.data)))
        return g

    def analyze(self, frame, min_points=16, closure_margin=8, frontier_only=True, queue_capacity=4096,
                pixel_budget=None, score_mode=0):
        p = capi.AnalysisParams()
        p.min_points = int(min_points)
        p.closure_margin = int(closure_margin)
        p.frontier_only = 1 if frontier_only else 0
        p.queue_capacity = int(queue_capacity)
        p.pixel_budget = float(frame.lod_pixel_budget if pixel_budget is None else pixel_budget)
        p.score_mode = int(score_mode)
        r = capi.AnalysisResult()
        self._ok(capi.lib().rb_analyze(self.h, ctypes.byref(frame), ctypes.byref(p), ctypes.byref(r)))
        return r

    def analysis(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_analysis(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=ANALYSIS_DTYPE)
        self._ok(capi.lib().rb_read_analysis(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n)))
        return out

    def queue(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_queue(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.uint32)
        if n.value:
            self._ok(capi.lib().rb_read_queue(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n)))
        return out

    def rollup(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_rollup(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 16), dtype=np.uint64)
        self._ok(capi.lib().rb_read_rollup(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n)))
        return out

    def features(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_features(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, capi.NUM_FEATURES), dtype=np.float32)
        self._ok(capi.lib().rb_read_features(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n)))
        return out

    def mlp_init(self, seed):
        self._ok(capi.lib().rb_mlp_init(self.h, int(seed)))

    def mlp_set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == capi.MLP_NUM_PARAMS
        self._ok(capi.lib().rb_mlp_set_params(self.h, ctypes.c_void_p(p.ctypes.data)))

    def mlp_params(self):
        p = np.zeros(capi.MLP_NUM_PARAMS, dtype=np.float32)
        self._ok(capi.lib().rb_mlp_get_params(self.h, ctypes.c_void_p(p.ctypes.data)))
        return p

    def mlp_predict(self, x_dev, y_dev):
        self._ok(capi.lib().rb_mlp_predict(self.h, x_dev.data_ptr(), int(x_dev.shape[0]), y_dev.data_ptr()))

    def mlp_gradients(self, x_dev, t_dev):
        g = np.zeros(capi.MLP_NUM_PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        self._ok(capi.lib().rb_mlp_gradients(self.h, x_dev.data_ptr(), t_dev.data_ptr(), int(x_dev.shape[0]),
                                             ctypes.c_void_p(g.ctypes.data), ctypes.byref(loss)))
        return g, loss.value

    def mlp_train_step(self, x_dev, t_dev, lr, want_loss=False):
        loss = ctypes.c_float()
        self._ok(capi.lib().rb_mlp_train_step(self.h, x_dev.data_ptr(), t_dev.data_ptr(), int(x_dev.shape[0]),
                                              float(lr), ctypes.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def refine(self, budget, mask):
        self._ok(capi.lib().rb_refine(self.h, int(budget), mask.data_ptr()))

    def refine_colors(self, budget):
        """Colour filtering of the first `budget` queued nodes' voxels (rb_refine_colors)."""
        r = capi.RefineResult()
        self._ok(capi.lib().rb_refine_colors(self.h, int(budget), ctypes.byref(r)))
        return r

    def refine_deepen(self, budget, min_points=0):
        """Deepening of the queued leaves among the first `budget` queue entries
        (rb_refine_deepen): split and their points redistributed."""
        r = capi.DeepenResult()
        self._ok(capi.lib().rb_refine_deepen(self.h, int(budget), int(min_points), ctypes.byref(r)))
        return r

    def refine_collapse(self, nodes, max_points=0):
        """Collapsing of the given nodes whose children are all leaves
        (rb_refine_collapse): each becomes a leaf with its children's points."""
        arr = np.ascontiguousarray(nodes, dtype=np.uint32)
        r = capi.CollapseResult()
        self._ok(capi.lib().rb_refine_collapse(self.h, ctypes.c_void_p(arr.ctypes.data) if len(arr) else None,
                                               len(arr), int(max_points), ctypes.byref(r)))
        return r

    def set_stream(self, stream_handle):
        self._ok(capi.lib().rb_set_stream(self.h, ctypes.c_void_p(int(stream_handle))))

    def set_profiling(self, on):
        self._ok(capi.lib().rb_set_profiling(self.h, 1 if on else 0))

    def reset_profile(self):
        self._ok(capi.lib().rb_reset_profile(self.h))

    def profile(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_profile(self.h, None, 0, ctypes.byref(n)))
        arr = (capi.KernelProfile * n.value)()
        self._ok(capi.lib().rb_read_profile(self.h, ctypes.cast(arr, ctypes.c_void_p), n.value, ctypes.byref(n)))
        return {k.name.decode(): {"launches": k.launches, "timed": k.timed_launches, "ms": k.total_ms,
                                  "units": k.units} for k in arr}

    def accums(self):
        n = ctypes.c_uint32()
        self._ok(capi.lib().rb_read_accums(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=ACCUM_DTYPE)
        self._ok(capi.lib().rb_read_accums(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n)))
        return out


class DeviceRing:
    """PointSource's device ring (include/remo/PointSource.h:69-115) over torch
    memory: `slots` slots of `slot_capacity` points; batch b lives in slot b % slots."""

    def __init__(self, points, batch_size, slots=50, slot_capacity=1000000, device="cuda"):
        import torch
        n = len(points)
        self.num_batches = (n + batch_size - 1) // batch_size
        self.slots = slots
        self.slot_capacity = slot_capacity
        self.ring = torch.zeros((slots, slot_capacity, 4), dtype=torch.float32, device=device)
        self.sizes = [0] * slots
        self.points = points
        self.batch_size = batch_size
        self.uploaded = 0

    def upload(self, b):
        import torch
        first = b * self.batch_size
        cnt = min(self.batch_size, len(self.points) - first)
        slot = b % self.slots
        host = np.ascontiguousarray(self.points[first:first + cnt]).view(np.float32).reshape(cnt, 4)
        self.ring[slot, :cnt].copy_(torch.from_numpy(host))
        self.sizes[slot] = cnt
        self.uploaded = b + 1

    def upload_window(self, consumed):
        """The producer window min(total, consumed + slots) (src/io/PointSource.cpp:223-239)."""
        while self.uploaded < min(self.num_batches, consumed + self.slots):
            self.upload(self.uploaded)
