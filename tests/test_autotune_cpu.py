"""Argument checks of the batch autotuner (dgmr_batch_autotune) and of the
batch view's blend block, on a host without a GPU: every call below is
answered before any CUDA work."""
import ctypes as C

import pytest

from differentiable_gaussian_mixture_renderer_b200 import _native as N


def _call(lib, kind=N.SERVE_SPLAT, n_views=2, depths=(1, 2), blocks=(8, 16), reps=1, view_scene=0, with_ms=True):
    scenes = (N.Scene * 1)()
    views = (N.BatchView * max(n_views, 1))()
    for v in views:
        v.scene = view_scene
    d = (C.c_int32 * len(depths))(*depths)
    b = (C.c_int32 * len(blocks))(*blocks)
    ms = (C.c_float * max(len(depths) * len(blocks), 1))()
    bd, bb = C.c_int32(0), C.c_int32(0)
    return lib.dgmr_batch_autotune(kind, scenes, 1, views, n_views, None, d, len(depths), b, len(blocks), reps, None, 0,
                                   None, 0, 0, ms if with_ms else None, C.byref(bd), C.byref(bb), None)


@pytest.mark.parametrize("args", [
    dict(kind=7),  # neither renderer
    dict(n_views=0),
    dict(n_views=N.BATCH_MAX_VIEWS + 1),
    dict(depths=(0,)),  # a batch holds at least one view
    dict(depths=()),
    dict(blocks=(32,)),  # the splat blend's blocks are 8x8 or 16x16 (0: the default)
    dict(kind=N.SERVE_MARCH, blocks=(8,)),  # the marcher has no blend block
    dict(reps=0),
    dict(view_scene=3),  # a view of a scene that is not there
    dict(with_ms=False),
])
def test_autotune_refuses_bad_arguments(args):
    lib = N.load()
    assert _call(lib, **args) == N.DGMR_ERR_BAD_ARG


def _size_query(lib, blocks):
    """dgmr_splat_batch_workspace_size for one float32 scene of 10 Gaussians
    (host addresses suffice: the query reads no tensor) and one view per entry
    of ``blocks``."""
    scene = (N.Scene * 1)()
    scene[0].dtype = N.DGMR_F32
    scene[0].n_gaussians = 10
    scene[0].sh_stride = 1
    dummy = (C.c_float * 160)()
    for f in ("centroids", "sh", "weights", "scales", "rotations"):
        setattr(scene[0], f, C.cast(dummy, C.c_void_p))
    views = (N.BatchView * len(blocks))()
    for v, b in zip(views, blocks):
        v.scene = 0
        v.blend_block = b
        v.camera = N.make_camera([1.0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 3, 1], [1.0] * 16, [0.0, 0.0, -3.0],
                                 (0.0, 0.0, 0.0), 64, 48, 0.5, 0.4)
    fb, pb = C.c_size_t(0), C.c_size_t(0)
    return lib.dgmr_splat_batch_workspace_size(scene, 1, views, len(blocks), 1000, C.byref(fb), C.byref(pb))


@pytest.mark.parametrize("blocks,ok", [
    ((0,), True), ((8,), True), ((16,), True), ((8, 0, 8), True),  # later views: 0 or the first view's side
    ((32,), False), ((4,), False), ((8, 16), False), ((0, 8), False),
])
def test_batch_blend_block_is_checked(blocks, ok):
    """dgmr_batch_view.blend_block: 0 (the library's choice), 8 or 16, the first
    view's value for the whole batch; anything else is refused before any work."""
    lib = N.load()
    st = _size_query(lib, blocks)
    assert (st == N.DGMR_OK) == ok, st
    if not ok:
        assert st == N.DGMR_ERR_BAD_ARG
