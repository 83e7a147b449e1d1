"""The C-ABI library loads on a CPU-only host and exports every symbol the
public header declares."""
import ctypes
import os
import re

from differentiable_gaussian_mixture_renderer_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(dgmr_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "dgmr_splat_forward" in names and "dgmr_vm_backward" in names
    assert set(names) == set(_native._SIGNATURES), "ctypes table out of sync with include/"


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_workspace_queries_without_gpu():
    lib = _native.load()
    assert lib.dgmr_splat_frame_workspace_size(1000, 256, 256) > 0
    assert lib.dgmr_splat_pair_workspace_size(1000, 5000) > lib.dgmr_splat_pair_workspace_size(1000, 100)
    assert lib.dgmr_splat_frame_workspace_size(-1, 256, 256) == 0
    assert lib.dgmr_vm_workspace_size(1000, 64, 64, 10, 1) > lib.dgmr_vm_workspace_size(1000, 64, 64, 10, 0)
    assert lib.dgmr_version().decode().startswith("dgmr_b200")
    assert lib.dgmr_status_string(2).decode() == "workspace too small"


def test_bad_arguments_are_rejected_on_the_host():
    lib = _native.load()
    scene = _native.Scene()
    cam = _native.Camera()
    cam.width, cam.height = 16, 16
    scene.n_gaussians, scene.sh_stride, scene.sh_degree, scene.dtype = 1, 0, 0, 0
    assert lib.dgmr_splat_forward(scene, cam, None, None, 0, None, 0, 0, None, None) == _native.DGMR_ERR_BAD_ARG
    scene.sh_stride = 1
    assert lib.dgmr_splat_forward(scene, cam, None, None, 0, None, 0, 0, None, None) == _native.DGMR_ERR_BAD_ARG
    assert lib.dgmr_vm_set_const_samples(5, None) == _native.DGMR_ERR_BAD_ARG
