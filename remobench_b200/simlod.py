"""The .simlod point-cloud file (src/io/RawReader.h:10-16) from Python: a
24-byte header of six floats (a box the loader never trusts) and then 16-byte
points {float x, y, z; uint32 rgba}. The C++ host reads the same files
(remobench_b200/host/simlod_file.cpp) and streams them through its point
source; this module writes them and reads them the same way: the observed box,
points translated to its minimum in float arithmetic
(src/io/PointSource.cpp:360-379).
"""
import os

import numpy as np

POINT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("color", "<u4")])
HEADER_BYTES = 24


def write(path, points, header_box=None):
    """Writes points (POINT_DTYPE) after a header box (default: their float bounds)."""
    pts = np.ascontiguousarray(points, dtype=POINT_DTYPE)
    if header_box is None:
        xyz = np.stack([pts["x"], pts["y"], pts["z"]], 1)
        header_box = np.concatenate([xyz.min(0), xyz.max(0)]) if len(pts) else np.zeros(6)
    with open(path, "wb") as f:
        f.write(np.asarray(header_box, dtype="<f4").tobytes())
        f.write(pts.tobytes())


def header(path):
    """(num_points, header_box); ValueError on a file that is not a whole
    number of points after the header, or holds none."""
    size = os.path.getsize(path)
    if size < HEADER_BYTES:
        raise ValueError(f"{path} is shorter than the 24-byte .simlod header")
    payload = size - HEADER_BYTES
    if payload % 16:
        raise ValueError(f"{path}: {payload} bytes after the header is not a whole number of 16-byte points")
    if payload == 0:
        raise ValueError(f"{path} has a header and no points")
    with open(path, "rb") as f:
        box = np.frombuffer(f.read(HEADER_BYTES), dtype="<f4").copy()
    return payload // 16, box


def points(path, first=0, count=None):
    """A memory map of points [first, first + count) as stored."""
    n, _ = header(path)
    if count is None:
        count = n - first
    if first < 0 or count < 0 or first + count > n:
        raise ValueError(f"points [{first}, {first + count}) lie past the {n} points of {path}")
    return np.memmap(path, dtype=POINT_DTYPE, mode="r", offset=HEADER_BYTES + 16 * first, shape=(count,))


def bounds(path):
    """The observed bounds (min xyz, max xyz) in float64."""
    p = points(path)
    lo, hi = [], []
    for a in "xyz":
        v = np.asarray(p[a], dtype=np.float64)
        lo.append(v.min())
        hi.append(v.max())
    return np.array(lo + hi)


def load(path, first=0, count=None):
    """(points translated to the observed minimum, box_min, box_max) as the
    octree sees them: box [0, size] in float32, coordinates + float(-min)."""
    b = bounds(path)
    t = (-b[:3]).astype(np.float32)
    p = np.array(points(path, first, count))
    if np.any(t != 0):
        for i, a in enumerate("xyz"):
            p[a] = p[a] + t[i]
    size = (b[3:] - b[:3]).astype(np.float32)
    return p, np.zeros(3, np.float32), size
