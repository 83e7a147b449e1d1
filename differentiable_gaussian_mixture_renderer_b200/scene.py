"""Seeded synthetic scenes and pinhole cameras in the reference's conventions.

No dataset is named for this path; benchmarks and tests use Gaussians drawn
as follows (all float32):

* centroids uniform in [-extent, extent]^3
* per-axis scales log-uniform in [0.005, 0.05]
* rotations: normalised N(0,1)^4, stored (w, x, y, z) -- the reference builds
  with GLM_FORCE_QUAT_DATA_WXYZ (python_bindings/util.py:77-86)
* weights (opacity) = sigmoid(N(0,1)), passed as is (the reference applies no
  activation)
* colours uniform in [0,1], encoded as the SH DC term (rgb - 0.5) / SH_C0

Cameras are OpenCV-style (x right, y down, +z forward; view-space z is the
depth the preprocess culls at 0.2).  ``view`` and ``proj`` are returned the way
the reference's torch binding receives them: the TRANSPOSE of the
mathematical matrix, so that reading torch row i as glm column i
(python_bindings/vol_marcher.cu:32-40) rebuilds the matrix.  ``proj`` is the
full view-projection P*V, with clip w = view-space z.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SH_C0 = 0.28209479177387814


@dataclass
class Scene:
    centroids: np.ndarray  # [N,3]
    sh: np.ndarray  # [N,k,3]
    weights: np.ndarray  # [N]
    scales: np.ndarray  # [N,3]
    rotations: np.ndarray  # [N,4] wxyz
    sh_degree: int = 0
    formulation: str | None = None  # None = the renderer's default; else opacity/mass/density/ots/ols

    @property
    def n(self) -> int:
        return int(self.centroids.shape[0])


@dataclass
class Camera:
    width: int
    height: int
    view: np.ndarray  # [4,4] torch layout (transposed)
    proj: np.ndarray  # [4,4] torch layout (transposed), full view-projection
    campos: np.ndarray  # [3]
    tan_fovx: float
    tan_fovy: float

    def astype(self, dtype) -> "Camera":
        return Camera(self.width, self.height, self.view.astype(dtype), self.proj.astype(dtype),
                      self.campos.astype(dtype), self.tan_fovx, self.tan_fovy)


def make_scene(n: int, seed: int = 0, extent: float = 1.0, sh_degree: int = 0,
               scale_range=(0.005, 0.05), dtype=np.float32) -> Scene:
    rng = np.random.default_rng(seed)
    centroids = rng.uniform(-extent, extent, size=(n, 3))
    lo, hi = math.log(scale_range[0]), math.log(scale_range[1])
    scales = np.exp(rng.uniform(lo, hi, size=(n, 3)))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    weights = 1.0 / (1.0 + np.exp(-rng.normal(size=n)))
    rgb = rng.uniform(0.0, 1.0, size=(n, 3))
    k = (sh_degree + 1) ** 2
    sh = np.zeros((n, k, 3))
    sh[:, 0, :] = (rgb - 0.5) / SH_C0
    if k > 1:
        sh[:, 1:, :] = rng.normal(scale=0.1, size=(n, k - 1, 3))
    f = lambda a: np.ascontiguousarray(a, dtype=dtype)
    return Scene(f(centroids), f(sh), f(weights), f(scales), f(q), sh_degree)


def look_at(eye, target, down_hint=(0.0, -1.0, 0.0)) -> np.ndarray:
    """World-to-view rotation+translation (math layout, 4x4, float64)."""
    eye = np.asarray(eye, dtype=np.float64)
    fwd = np.asarray(target, dtype=np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    d = np.asarray(down_hint, dtype=np.float64)
    if abs(np.dot(d, fwd)) > 0.99:
        d = np.array([0.0, 0.0, 1.0])
    right = np.cross(d, fwd)
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = right, down, fwd
    V[:3, 3] = -V[:3, :3] @ eye
    return V


def perspective(tan_fovx: float, tan_fovy: float, znear=0.01, zfar=100.0) -> np.ndarray:
    P = np.zeros((4, 4))
    P[0, 0] = 1.0 / tan_fovx
    P[1, 1] = 1.0 / tan_fovy
    P[2, 2] = zfar / (zfar - znear)
    P[2, 3] = -(zfar * znear) / (zfar - znear)
    P[3, 2] = 1.0
    return P


def make_camera(width: int, height: int, eye=(0.0, 0.0, -3.0), target=(0.0, 0.0, 0.0),
                fovy_deg: float = 60.0, dtype=np.float32) -> Camera:
    tan_fovy = math.tan(math.radians(fovy_deg) * 0.5)
    tan_fovx = tan_fovy * width / height
    V = look_at(eye, target)
    P = perspective(tan_fovx, tan_fovy)
    full = P @ V
    return Camera(width, height, np.ascontiguousarray(V.T, dtype=dtype),
                  np.ascontiguousarray(full.T, dtype=dtype),
                  np.asarray(eye, dtype=dtype), float(np.float32(tan_fovx)), float(np.float32(tan_fovy)))


def random_cameras(count: int, width: int, height: int, seed: int = 1,
                   radius=(2.5, 4.0), dtype=np.float32) -> list[Camera]:
    """Cameras on a sphere around the origin, looking at it."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(count):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        r = rng.uniform(*radius)
        cams.append(make_camera(width, height, eye=tuple(d * r), dtype=dtype))
    return cams
