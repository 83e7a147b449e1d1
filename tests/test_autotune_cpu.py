"""The batch autotuner's argument checks (dgmr_batch_autotune), on a host
without a GPU: every call below is refused before any CUDA work."""
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
