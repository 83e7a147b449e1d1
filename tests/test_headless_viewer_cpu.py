"""The headless viewer and its C++ interface without a GPU: the file formats
round-trip, the interface header compiles as plain C++17, and the viewer
rejects bad command lines and files before touching a device."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from differentiable_gaussian_mixture_renderer_b200 import build, headless, scene as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def viewer():
    return build.build_viewer()


def test_scene_and_camera_files_round_trip(tmp_path):
    sc = S.make_scene(37, seed=2, sh_degree=2)
    headless.write_scene(str(tmp_path / "s.bin"), sc)
    back = headless.read_scene(str(tmp_path / "s.bin"))
    assert back["sh_degree"] == 2
    for k in ("centroids", "sh", "weights", "scales", "rotations"):
        np.testing.assert_array_equal(back[k], np.asarray(getattr(sc, k), np.float32).reshape(back[k].shape))
    cam = S.make_camera(40, 30)
    headless.write_camera(str(tmp_path / "c.bin"), cam)
    data = (tmp_path / "c.bin").read_bytes()
    assert data[:8] == b"DGMRCAM1" and struct.unpack_from("<2i", data, 8) == (40, 30)
    assert len(data) == 16 + 4 * (16 + 16 + 3 + 2)
    view = np.frombuffer(data, "<f4", 16, 16)
    np.testing.assert_array_equal(view, cam.view.reshape(16))


def test_ppm_conversion_rounds_half_up_and_clamps():
    fb = np.array([-1.0, 0.0, 0.5 / 255, 0.25, 0.5, 1.0, 2.0, np.nan], np.float32)
    fb = np.stack([fb, fb, fb]).reshape(3, 1, 8)
    px = headless.to_ppm_bytes(fb)[0, :, 0]
    assert list(px) == [0, 0, 1, 64, 128, 255, 255, 0]


def test_interface_header_compiles_as_cxx17(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    cuda_inc = "/usr/local/cuda/include"
    if not cxx or not os.path.exists(os.path.join(cuda_inc, "cuda_runtime.h")):
        pytest.skip("no host C++ compiler or CUDA headers")
    src = tmp_path / "use.cpp"
    src.write_text('#include "dgmr_b200_sibr.hpp"\n'
                   'int main() { dgmr_b200::SplatForwardData d; d.sh_degree = 0; '
                   'dgmr_b200::VolMarcherForwardData m; return m.debug_render_bin == -1 && d.sh_stride == 16 ? 0 : 1; }\n')
    subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    "-I", cuda_inc, str(src)], check=True)


def test_viewer_help_and_argument_errors(viewer, tmp_path):
    r = subprocess.run([viewer, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage" in r.stdout
    for args in ([], ["--scene", "x"], ["--scene", "x", "--camera", "y", "--renderer", "gl"],
                 ["--scene", "x", "--camera", "y", "--formulation", "foo"], ["--frames"],
                 ["--scene", "x", "--camera", "y", "--background", "1,2"]):
        r = subprocess.run([viewer, *args], capture_output=True, text=True)
        assert r.returncode == 2, (args, r.stderr)


def test_viewer_rejects_malformed_files(viewer, tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"DGMRSCN1" + struct.pack("<4i", 10, 1, 0, 0) + b"\0" * 12)  # truncated arrays
    cam = tmp_path / "c.bin"
    headless.write_camera(str(cam), S.make_camera(16, 16))
    r = subprocess.run([viewer, "--scene", str(bad), "--camera", str(cam)], capture_output=True, text=True)
    assert r.returncode == 2 and "malformed scene" in r.stderr
    good = tmp_path / "s.bin"
    headless.write_scene(str(good), S.make_scene(5, seed=1))
    cam.write_bytes(b"DGMRCAM1" + struct.pack("<2i", 0, 16))
    r = subprocess.run([viewer, "--scene", str(good), "--camera", str(cam)], capture_output=True, text=True)
    assert r.returncode == 2 and "malformed camera" in r.stderr
