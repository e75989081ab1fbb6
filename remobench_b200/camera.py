"""Seeded orbit cameras and projection matrices (headless).

Restates the reference's orbit controls (src/shell/OrbitControls.h:68-93:
world = T(target) Rz(yaw) Rx(pitch) flip T(0, 0, radius), view = world^-1) and
glm::perspective (src/shell/GLRenderer.cpp:77) with near = extent * 1e-4 and
far = extent * 100 (src/shell/App.cpp:205-209). Matrices are row-major,
clip = M (x, y, z, 1), computed in float64 and handed over as float32.
"""
import math

import numpy as np


def _translate(t):
    m = np.eye(4)
    m[:3, 3] = t
    return m


def _rotate(angle, axis):
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    c, s = math.cos(angle), math.sin(angle)
    x, y, z = a
    r = np.eye(4)
    r[:3, :3] = [[c + x * x * (1 - c), x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                 [y * x * (1 - c) + z * s, c + y * y * (1 - c), y * z * (1 - c) - x * s],
                 [z * x * (1 - c) - y * s, z * y * (1 - c) + x * s, c + z * z * (1 - c)]]
    return r


_FLIP = np.array([[1.0, 0.0, 0.0, 0.0],
                  [0.0, 0.0, -1.0, 0.0],
                  [0.0, 1.0, 0.0, 0.0],
                  [0.0, 0.0, 0.0, 1.0]])


def perspective(fovy, aspect, near, far):
    f = 1.0 / math.tan(fovy / 2.0)
    p = np.zeros((4, 4))
    p[0, 0] = f / aspect
    p[1, 1] = f
    p[2, 2] = -(far + near) / (far - near)
    p[2, 3] = -2.0 * far * near / (far - near)
    p[3, 2] = -1.0
    return p


class Orbit:
    """frameBox (OrbitControls.h:68-75) and update (:77-93)."""

    def __init__(self, box_min, box_max, fovy=math.radians(60.0)):
        bmin = np.asarray(box_min, dtype=np.float64)
        bmax = np.asarray(box_max, dtype=np.float64)
        self.target = (bmin + bmax) * 0.5
        extent = float(np.linalg.norm(bmax - bmin))
        self.radius = (extent * 0.5) / math.tan(max(fovy, 1e-3) * 0.5) * 1.1
        self.yaw = 0.35
        self.pitch = -0.6
        self.fovy = fovy
        ext = max(float(bmax[0] - bmin[0]), float(bmax[1] - bmin[1]), float(bmax[2] - bmin[2]), 1.0)
        self.near = ext * 1e-4
        self.far = ext * 100.0

    def world(self):
        return (_translate(self.target) @ _rotate(self.yaw, (0, 0, 1)) @ _rotate(self.pitch, (1, 0, 0))
                @ _FLIP @ _translate((0.0, 0.0, self.radius)))

    def view_proj(self, width, height):
        view = np.linalg.inv(self.world())
        return perspective(self.fovy, width / height, self.near, self.far) @ view


def orbit_path(box_min, box_max, frames, seed=0, fovy=math.radians(60.0)):
    """A seeded orbit: yaw sweeps a full turn, pitch and radius drift smoothly.
    Yields (yaw, pitch, radius_scale) per frame."""
    rng = np.random.default_rng(seed)
    p0, p1 = rng.uniform(-1.1, -0.35), rng.uniform(0.0, 2 * math.pi)
    r0, r1 = rng.uniform(0.35, 0.9), rng.uniform(0.0, 2 * math.pi)
    yaw0 = rng.uniform(0.0, 2 * math.pi)
    out = []
    for k in range(frames):
        t = k / max(frames, 1)
        out.append((yaw0 + 2 * math.pi * t, p0 + 0.15 * math.sin(2 * math.pi * t + p1),
                    r0 * (1.0 + 0.25 * math.sin(2 * math.pi * t + r1))))
    return out


def frame_matrices(box_min, box_max, width, height, yaw=None, pitch=None, radius_scale=1.0):
    o = Orbit(box_min, box_max)
    if yaw is not None:
        o.yaw = yaw
    if pitch is not None:
        o.pitch = pitch
    o.radius *= radius_scale
    return o.view_proj(width, height).astype(np.float32)
