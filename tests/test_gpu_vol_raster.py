"""vol_raster forward on the GPU against the CPU oracle (restating
src/dgmr/vol_raster_forward.cu:39-520)."""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import scene as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-4


def _run(sc, cam, bg, **kw):
    from differentiable_gaussian_mixture_renderer_b200 import vol_raster
    dev = torch.device("cuda:0")
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    return vol_raster.forward(t(sc.sh), t(sc.weights), t(sc.centroids), t(sc.scales), t(sc.rotations), t(cam.view),
                              t(cam.proj), t(cam.campos), t(np.array(bg, np.float32)), cam.width, cam.height,
                              cam.tan_fovx, cam.tan_fovy, sc.sh_degree, **kw)


@pytest.mark.parametrize("n,w,h,seed,deg", [(3000, 64, 48, 1, 0), (8000, 96, 80, 2, 1), (20000, 128, 128, 3, 2)])
def test_vol_raster_matches_oracle(cuda, n, w, h, seed, deg):
    sc = S.make_scene(n, seed=seed, sh_degree=deg)
    cam = S.random_cameras(1, w, h, seed=seed + 40)[0]
    bg = (0.1, 0.2, 0.3)
    ref = O.vr_forward(sc, cam, bg=np.array(bg, np.float32))
    fb = _run(sc, cam, bg).cpu().numpy()
    assert np.isfinite(fb).all()
    err = float(np.abs(fb - ref["fb"]).max())
    assert err <= IMAGE_TOL, err


def test_vol_raster_empty_frame_and_bins_mode_are_background(cuda):
    sc = S.make_scene(500, seed=4)
    cam = S.make_camera(32, 32, eye=(0.0, 0.0, 3.0), target=(0.0, 0.0, 6.0))  # looking away from the scene
    bg = (0.25, 0.5, 0.75)
    fb = _run(sc, cam, bg).cpu().numpy()
    assert np.allclose(fb, np.array(bg, np.float32)[:, None, None])
    cam = S.make_camera(32, 32)
    fb = _run(sc, cam, bg, render_mode="bins").cpu().numpy()
    assert np.allclose(fb, np.array(bg, np.float32)[:, None, None])


def test_vol_raster_depth_mode(cuda):
    sc = S.make_scene(4000, seed=5)
    cam = S.make_camera(48, 48)
    fb = _run(sc, cam, (0.0, 0.0, 0.0), render_mode="depth", max_depth=10.0).cpu().numpy()
    covered = fb[1] != 1.0  # pixels whose last bin ends at 0 are drawn green (0, 1, 0)
    assert covered.any()
    # grey depth in the covered pixels: the last bin's end over max_depth (camera at distance 3)
    d = fb[0][covered]
    assert np.allclose(fb[0][covered], fb[2][covered]) and (d > 0.1).all() and (d < 1.0).all()
