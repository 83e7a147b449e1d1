"""The C-ABI library loads on a CPU-only host and exports every symbol the
public header declares."""
import ctypes
import os
import re

import pytest

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
    # the marcher's backward accumulators are double for both dtypes: 13 x 8 bytes per Gaussian at least
    assert lib.dgmr_vm_workspace_size(1000, 64, 64, 10, 1) >= lib.dgmr_vm_workspace_size(1000, 64, 64, 10, 0) > 1000 * 13 * 8
    assert lib.dgmr_vm_workspace_size(1000, 64, 64, 5000, 0) > lib.dgmr_vm_workspace_size(1000, 64, 64, 10, 0)
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


def test_scene_struct_layout_and_formulation_codes():
    import ctypes as C
    import pytest
    # dgmr_scene: 4 int32, 5 pointers, formulation, reserved
    assert C.sizeof(_native.Scene) == 64 and _native.Scene.formulation.offset == 56
    assert [_native.formulation_code(f) for f in (None, "opacity", "Mass", "density", "ots", "OLS", 3)] == \
        [0, 1, 2, 3, 4, 5, 3]
    for bad in ("gaussian", 6, -1, True, 1.0):
        with pytest.raises(ValueError):
            _native.formulation_code(bad)
    lib = _native.load()
    scene = _native.Scene()
    cam = _native.Camera()
    cam.width, cam.height = 16, 16
    scene.n_gaussians, scene.sh_stride, scene.sh_degree, scene.dtype = 0, 1, 0, 0
    scene.formulation = 6  # out of range: rejected before any device work
    assert lib.dgmr_splat_forward(scene, cam, None, None, 0, None, 0, 0, None, None) == _native.DGMR_ERR_BAD_ARG


def _batch_tables(n_views, scene_index=0, n_scenes=1):
    scenes = (_native.Scene * n_scenes)()
    for s in scenes:
        s.n_gaussians, s.sh_stride, s.sh_degree, s.dtype = 1000, 1, 0, 0
        s.centroids = s.sh = s.weights = s.scales = s.rotations = 4096  # never dereferenced by the size query
    views = (_native.BatchView * n_views)()
    for k, v in enumerate(views):
        v.scene = scene_index
        v.camera.width, v.camera.height = 64 + 16 * k, 48
        for i in (0, 5, 10, 15):
            v.camera.view[i] = v.camera.proj[i] = 1.0
        v.camera.tan_fovx = v.camera.tan_fovy = 0.5
    return scenes, views


@pytest.mark.parametrize("prefix", ["dgmr_splat_batch_", "dgmr_vm_batch_"])
def test_batch_workspace_query_without_gpu(prefix):
    import ctypes as C
    lib = _native.load()
    size = getattr(lib, prefix + "workspace_size")
    fb, pb = C.c_size_t(0), C.c_size_t(0)
    scenes, views = _batch_tables(3)
    assert size(scenes, 1, views, 3, 1000, C.byref(fb), C.byref(pb)) == 0
    three = (fb.value, pb.value)
    scenes, views = _batch_tables(6)
    assert size(scenes, 1, views, 6, 1000, C.byref(fb), C.byref(pb)) == 0
    assert fb.value > three[0]  # twice the view-Gaussian slots
    assert size(scenes, 1, views, 6, 100000, C.byref(fb), C.byref(pb)) == 0
    assert pb.value > three[1]


@pytest.mark.parametrize("prefix", ["dgmr_splat_batch_", "dgmr_vm_batch_"])
def test_batch_bad_arguments_without_gpu(prefix):
    import ctypes as C
    lib = _native.load()
    size = getattr(lib, prefix + "workspace_size")
    fb, pb = C.c_size_t(0), C.c_size_t(0)
    scenes, views = _batch_tables(2, scene_index=1)  # scene index out of range
    assert size(scenes, 1, views, 2, 0, C.byref(fb), C.byref(pb)) == _native.DGMR_ERR_BAD_ARG
    scenes, views = _batch_tables(_native.BATCH_MAX_VIEWS + 1)
    assert size(scenes, 1, views, _native.BATCH_MAX_VIEWS + 1, 0, C.byref(fb), C.byref(pb)) == _native.DGMR_ERR_BAD_ARG
    scenes, views = _batch_tables(2)
    scenes[0].dtype = 1  # float64: batches are float32 only
    assert size(scenes, 1, views, 2, 0, C.byref(fb), C.byref(pb)) == _native.DGMR_ERR_BAD_ARG
    scenes, views = _batch_tables(2)
    assert getattr(lib, prefix + "forward")(scenes, 1, views, 2, None, 0, None, 0, 0, None, None) == _native.DGMR_ERR_BAD_ARG
    tail = [None] if prefix == "dgmr_vm_batch_" else []  # the marcher's backward also takes stats
    assert getattr(lib, prefix + "backward")(scenes, 1, views, 2, None, None, 0, None, 0, 0, *tail,
                                             None) == _native.DGMR_ERR_BAD_ARG


def test_server_entry_points_without_gpu():
    """The native server's argument checks run on the host; without a device
    dgmr_server_create reports DGMR_ERR_CUDA instead of crashing."""
    import ctypes as C
    lib = _native.load()
    assert lib.dgmr_server_create(None, None) == _native.DGMR_ERR_BAD_ARG
    handle = C.c_void_p()
    cfg = _native.ServerConfig(0, 4, 8, 0, 0, 1.3)
    st = lib.dgmr_server_create(C.byref(cfg), C.byref(handle))
    if st == _native.DGMR_OK:  # a GPU is present: exercise the host-side checks, then release it
        req = _native.ServerRequest()
        assert lib.dgmr_server_submit(handle, C.byref(req)) == _native.DGMR_ERR_BAD_ARG  # no scene, no framebuffer
        assert lib.dgmr_server_poll(handle, None, 0) == 0 and lib.dgmr_server_pending(handle) == 0
        assert lib.dgmr_server_destroy(handle) == _native.DGMR_OK
    else:
        assert st == _native.DGMR_ERR_CUDA and not handle.value
    assert lib.dgmr_server_submit(None, None) == _native.DGMR_ERR_BAD_ARG
    assert lib.dgmr_server_poll(None, None, 0) == -1 and lib.dgmr_server_wait(None, None, 0) == -1
    assert lib.dgmr_server_pending(None) == -1
    assert lib.dgmr_server_get_stats(None, None) == _native.DGMR_ERR_BAD_ARG
    assert lib.dgmr_server_destroy(None) == _native.DGMR_ERR_BAD_ARG
    scene = _native.Scene()
    scene.dtype = 1  # float64 scenes are not served
    idx = C.c_int32()
    assert lib.dgmr_server_add_scene(None, C.byref(scene), C.byref(idx)) == _native.DGMR_ERR_BAD_ARG
