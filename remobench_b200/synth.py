"""Seeded synthetic lidar clouds (binding of csrc/synth.c, built into lib/librb_synth.so)."""
import ctypes
import os

import numpy as np

_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "librb_synth.so")

POINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("color", "<u4")])


class SynthConfig(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("num_points", ctypes.c_uint64),
        ("batch_size", ctypes.c_uint32),
        ("num_boxes", ctypes.c_uint32),
        ("num_poles", ctypes.c_uint32),
        ("num_threads", ctypes.c_uint32),
        ("tile", ctypes.c_double),
        ("origin_x", ctypes.c_double),
        ("origin_y", ctypes.c_double),
        ("outlier_fraction", ctypes.c_double),
        ("range_noise", ctypes.c_double),
        ("quantum", ctypes.c_double),
    ]


class SceneInfo(ctypes.Structure):
    _fields_ = [
        ("box_min", ctypes.c_double * 3),
        ("box_max", ctypes.c_double * 3),
        ("num_lanes", ctypes.c_uint32),
        ("sensor_height", ctypes.c_double),
    ]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise RuntimeError(f"{_LIB} is missing: run remobench_b200.build.build_all()")
        L = ctypes.CDLL(_LIB)
        L.rb_synth_default_config.argtypes = [ctypes.c_int, ctypes.POINTER(SynthConfig)]
        L.rb_synth_scene_info_get.argtypes = [ctypes.POINTER(SynthConfig), ctypes.POINTER(SceneInfo)]
        L.rb_synth_generate.argtypes = [ctypes.POINTER(SynthConfig), ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.c_int, ctypes.c_void_p]
        L.rb_synth_generate_f64.argtypes = [ctypes.POINTER(SynthConfig), ctypes.c_uint64,
                                            ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def config(config_id, **overrides):
    """Default configuration 1, 2, 3 or 5, with field overrides."""
    c = SynthConfig()
    if _load().rb_synth_default_config(int(config_id), ctypes.byref(c)) != 0:
        raise ValueError(f"unknown synthetic configuration {config_id}")
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


def scene_box(cfg, relative=True):
    """(box_min, box_max) of the cloud as float32 triples; relative to the box minimum
    when relative, as the reference's readers translate (src/io/PointSource.cpp:355-365)."""
    info = SceneInfo()
    if _load().rb_synth_scene_info_get(ctypes.byref(cfg), ctypes.byref(info)) != 0:
        raise RuntimeError("scene construction failed")
    lo = [float(v) for v in info.box_min]
    hi = [float(v) for v in info.box_max]
    if relative:
        hi = [h - l for h, l in zip(hi, lo)]
        lo = [0.0, 0.0, 0.0]
    return (np.array(lo, dtype=np.float32), np.array(hi, dtype=np.float32))


def scene_box_f64(cfg):
    """(box_min, box_max) of the cloud in float64 world coordinates."""
    info = SceneInfo()
    if _load().rb_synth_scene_info_get(ctypes.byref(cfg), ctypes.byref(info)) != 0:
        raise RuntimeError("scene construction failed")
    return (np.array([float(v) for v in info.box_min], dtype=np.float64),
            np.array([float(v) for v in info.box_max], dtype=np.float64))


def generate(cfg, first=0, count=None, relative=True, out=None):
    """Points [first, first+count) as a structured float32/uint32 array."""
    if count is None:
        count = cfg.num_points - first
    if out is None:
        out = np.empty(count, dtype=POINT_DTYPE)
    if out.dtype != POINT_DTYPE or len(out) < count or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous POINT_DTYPE array")
    rc = _load().rb_synth_generate(ctypes.byref(cfg), first, count, 1 if relative else 0,
                                   ctypes.c_void_p(out.ctypes.data))
    if rc != 0:
        raise ValueError("rb_synth_generate rejected the request (first must be batch-aligned)")
    return out


def generate_f64(cfg, first=0, count=None):
    """World coordinates in float64 (N x 3) and colours."""
    if count is None:
        count = cfg.num_points - first
    xyz = np.empty((count, 3), dtype=np.float64)
    col = np.empty(count, dtype=np.uint32)
    rc = _load().rb_synth_generate_f64(ctypes.byref(cfg), first, count,
                                       ctypes.c_void_p(xyz.ctypes.data), ctypes.c_void_p(col.ctypes.data))
    if rc != 0:
        raise ValueError("rb_synth_generate_f64 rejected the request")
    return xyz, col
