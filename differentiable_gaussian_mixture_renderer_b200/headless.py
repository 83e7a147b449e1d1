"""Files and launcher of the headless viewer (viewer/headless_view.cpp), the
C++ caller of the viewer interface include/dgmr_b200_sibr.hpp (the
reference's sibr_interfaces, src/dgmr/sibr_interfaces.cpp:26-44, without a
window).

Scene file: b"DGMRSCN1", int32 n, sh_stride, sh_degree, reserved, then
float32 centroids [n,3], sh [n,sh_stride,3], weights [n], scales [n,3],
rotations [n,4] (w,x,y,z).  Camera file: b"DGMRCAM1", int32 width, height,
float32 view[16], proj[16] (glm order: the row-major bytes of the transposed
torch matrices), campos[3], tan_fovx, tan_fovy.  All little endian.
"""
from __future__ import annotations

import os
import struct
import subprocess

import numpy as np

SCENE_MAGIC = b"DGMRSCN1"
CAMERA_MAGIC = b"DGMRCAM1"


def _f32(a) -> bytes:
    return np.ascontiguousarray(a, dtype="<f4").tobytes()


def write_scene(path: str, scene) -> None:
    """scene: an object with centroids, sh, weights, scales, rotations and
    sh_degree (scene.Scene or serving.GaussianScene moved to the host)."""
    sh = np.asarray(scene.sh, dtype=np.float32)
    n = int(np.asarray(scene.centroids).shape[0])
    if sh.ndim != 3 or sh.shape[0] != n or sh.shape[2] != 3 or not 1 <= sh.shape[1] <= 16:
        raise ValueError("sh must be [n, k<=16, 3]")
    with open(path, "wb") as f:
        f.write(SCENE_MAGIC + struct.pack("<4i", n, sh.shape[1], int(scene.sh_degree), 0))
        for a, shape in ((scene.centroids, (n, 3)), (sh, sh.shape), (np.asarray(scene.weights).reshape(-1), (n,)),
                         (scene.scales, (n, 3)), (scene.rotations, (n, 4))):
            a = np.asarray(a, dtype=np.float32)
            if a.shape != shape:
                raise ValueError(f"array of shape {a.shape}, expected {shape}")
            f.write(_f32(a))


def read_scene(path: str) -> dict:
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != SCENE_MAGIC:
        raise ValueError("not a scene file")
    n, k, deg, _ = struct.unpack_from("<4i", data, 8)
    off = 24
    out = {"sh_degree": deg}
    for name, shape in (("centroids", (n, 3)), ("sh", (n, k, 3)), ("weights", (n,)), ("scales", (n, 3)),
                        ("rotations", (n, 4))):
        count = int(np.prod(shape))
        out[name] = np.frombuffer(data, dtype="<f4", count=count, offset=off).reshape(shape)
        off += 4 * count
    if off != len(data):
        raise ValueError("trailing bytes in scene file")
    return out


def write_camera(path: str, cam) -> None:
    """cam: scene.Camera (view / proj already in the transposed torch layout)."""
    with open(path, "wb") as f:
        f.write(CAMERA_MAGIC + struct.pack("<2i", int(cam.width), int(cam.height)))
        f.write(_f32(np.asarray(cam.view).reshape(16)) + _f32(np.asarray(cam.proj).reshape(16)))
        f.write(_f32(np.asarray(cam.campos).reshape(3)) + _f32([cam.tan_fovx, cam.tan_fovy]))


def read_raw(path: str, width: int, height: int) -> np.ndarray:
    return np.fromfile(path, dtype="<f4").reshape(3, height, width)


def read_ppm(path: str) -> np.ndarray:
    """An 8-bit binary PPM as uint8 [H, W, 3]."""
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(maxsplit=4)
    if parts[0] != b"P6" or parts[3] != b"255":
        raise ValueError("not an 8-bit P6 image")
    w, h = int(parts[1]), int(parts[2])
    return np.frombuffer(parts[4][:w * h * 3], dtype=np.uint8).reshape(h, w, 3)


def to_ppm_bytes(fb: np.ndarray) -> np.ndarray:
    """The viewer's conversion of a [3,H,W] framebuffer to 8 bits: clamp to
    [0,1] (NaN to 0), times 255, rounded half away from zero."""
    v = np.nan_to_num(np.asarray(fb, dtype=np.float32), nan=0.0)
    v = np.clip(v, np.float32(0.0), np.float32(1.0)) * np.float32(255.0)  # float32 product, as in C++
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8).transpose(1, 2, 0)  # exact half-up


def viewer_path() -> str:
    from . import build
    return build.VIEWER_PATH


def run(scene_path: str, camera_path: str, renderer: str = "splat", frames: int = 1, ppm: str | None = None,
        raw: str | None = None, background=(0.0, 0.0, 0.0), formulation: str | None = None, mode: str = "full",
        debug_bin: int = -1, max_depth: float = 20.0, timeout: float = 600.0) -> dict:
    """Runs the viewer; returns its report line as a dict (renderer, frames,
    ms_per_frame, n_pairs, flags, width, height).  Raises CalledProcessError
    with the viewer's message on failure."""
    exe = viewer_path()
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} is not built (differentiable_gaussian_mixture_renderer_b200.build)")
    cmd = [exe, "--scene", scene_path, "--camera", camera_path, "--renderer", renderer, "--frames", str(frames),
           "--background", ",".join(repr(float(np.float32(b))) for b in background), "--mode", mode, "--bin",
           str(debug_bin), "--max-depth", repr(float(max_depth))]
    if formulation is not None:
        cmd += ["--formulation", formulation]
    if ppm:
        cmd += ["--ppm", ppm]
    if raw:
        cmd += ["--raw", raw]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout).stdout
    line = out.strip().splitlines()[-1]
    rep = dict(kv.split("=", 1) for kv in line.split())
    for k in ("frames", "n_pairs", "flags", "width", "height"):
        rep[k] = int(rep[k])
    rep["ms_per_frame"] = float(rep["ms_per_frame"])
    return rep
