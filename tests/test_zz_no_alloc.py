"""dgmr_splat_forward_noalloc: the splat forward for callers that cannot
allocate device memory (its workspaces live in a static device array inside
the library).  Called through the C ABI and compared with the workspace-taking
dgmr_splat_forward on two calls in a row -- different scenes and resolutions,
so anything the first call leaves in the shared array would show up in the
second.  Collected last so a failure here cannot hide the other results."""
import ctypes

import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import _native as N, scene as S

pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-4
STATIC_BYTES = 64 << 20


def _frame(n, w, h, seed, dev):
    sc = S.make_scene(n, seed=seed, sh_degree=1)
    cam = S.make_camera(w, h, eye=(0.2, -0.1, -3.0))
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    tensors = (t(sc.sh), t(sc.weights), t(sc.centroids), t(sc.scales), t(sc.rotations))
    scene = N.make_scene(*tensors, sc.sh_degree)
    camera = N.make_camera(cam.view, cam.proj, cam.campos, (0.1, 0.2, 0.3), w, h, cam.tan_fovx, cam.tan_fovy)
    return tensors, scene, camera


def _with_workspaces(lib, scene, camera, cap, dev):
    n, w, h = scene.n_gaussians, camera.width, camera.height
    fws = torch.empty(lib.dgmr_splat_frame_workspace_size(n, w, h), dtype=torch.uint8, device=dev)
    pws = torch.empty(max(1, lib.dgmr_splat_pair_workspace_size(n, cap)), dtype=torch.uint8, device=dev)
    fb = torch.empty((3, h, w), dtype=torch.float32, device=dev)
    stats = torch.zeros(4, dtype=torch.int32, device=dev)
    st = lib.dgmr_splat_forward(scene, camera, fb.data_ptr(), fws.data_ptr(), fws.numel(), pws.data_ptr(), pws.numel(),
                                cap, stats.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == N.DGMR_OK
    return fb, stats


def test_noalloc_forward_matches_workspace_forward_twice(cuda):
    lib = N.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for n, w, h, seed, cap in ((10000, 256, 256, 0, 60000), (3000, 200, 120, 7, 20000)):
        tensors, scene, camera = _frame(n, w, h, seed, cuda)
        assert lib.dgmr_splat_frame_workspace_size(n, w, h) + lib.dgmr_splat_pair_workspace_size(n, cap) < STATIC_BYTES
        ref, ref_stats = _with_workspaces(lib, scene, camera, cap, cuda)
        fb = torch.full((3, h, w), -1.0, dtype=torch.float32, device=cuda)
        stats = torch.zeros(4, dtype=torch.int32, device=cuda)
        st = lib.dgmr_splat_forward_noalloc(scene, camera, fb.data_ptr(), cap, stats.data_ptr(), stream)
        assert st == N.DGMR_OK, lib.dgmr_status_string(st)
        torch.cuda.synchronize()
        assert int(stats[1]) == 0 and int(ref_stats[1]) == 0
        assert int(stats[0]) == int(ref_stats[0]) > 0
        assert float((fb - ref).abs().max()) <= IMAGE_TOL


def test_noalloc_rejects_frames_beyond_the_static_scratch(cuda):
    lib = N.lib()
    n, w, h = 600_000, 64, 64
    assert lib.dgmr_splat_frame_workspace_size(n, w, h) > STATIC_BYTES
    tensors, scene, camera = _frame(n, w, h, 1, cuda)
    fb = torch.empty((3, h, w), dtype=torch.float32, device=cuda)
    st = lib.dgmr_splat_forward_noalloc(scene, camera, fb.data_ptr(), 1000, None,
                                        torch.cuda.current_stream().cuda_stream)
    assert st == N.DGMR_ERR_STATIC_SCRATCH
    assert b"static scratch" in lib.dgmr_status_string(st)


def test_noalloc_reports_a_too_small_pair_capacity(cuda):
    """With a device stats block the call stays asynchronous and flags the
    overflow there; without one it waits for the frame and returns
    DGMR_ERR_PAIR_OVERFLOW, so an incomplete image never passes as DGMR_OK."""
    lib = N.lib()
    stream = torch.cuda.current_stream().cuda_stream
    tensors, scene, camera = _frame(10000, 256, 256, 0, cuda)
    fb = torch.empty((3, 256, 256), dtype=torch.float32, device=cuda)
    stats = torch.zeros(4, dtype=torch.int32, device=cuda)
    assert lib.dgmr_splat_forward_noalloc(scene, camera, fb.data_ptr(), 100, stats.data_ptr(), stream) == N.DGMR_OK
    torch.cuda.synchronize()
    assert int(stats[1]) & 1 and int(stats[0]) > 100
    st = lib.dgmr_splat_forward_noalloc(scene, camera, fb.data_ptr(), 100, None, stream)
    assert st == N.DGMR_ERR_PAIR_OVERFLOW
    assert b"pair capacity" in lib.dgmr_status_string(st)
    # a sufficient capacity after the overflow: status OK and the full image
    cap = int(stats[0])
    ref, _ = _with_workspaces(lib, scene, camera, cap, cuda)
    assert lib.dgmr_splat_forward_noalloc(scene, camera, fb.data_ptr(), cap, None, stream) == N.DGMR_OK
    torch.cuda.synchronize()
    assert float((fb - ref).abs().max()) <= IMAGE_TOL
