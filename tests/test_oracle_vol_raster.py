"""The oracle's vol_raster restatement on the CPU: an empty frame is the
background, the image is finite, and more Gaussians in front never lighten a
black background (the blend only adds emission attenuated by transparency)."""
import numpy as np

from differentiable_gaussian_mixture_renderer_b200 import scene as S
from oracle import oracle as O


def test_empty_frame_is_background():
    sc = S.make_scene(300, seed=1)
    cam = S.make_camera(24, 16, eye=(0.0, 0.0, 3.0), target=(0.0, 0.0, 6.0))
    out = O.vr_forward(sc, cam, bg=np.array([0.2, 0.4, 0.6], np.float32))
    assert out["n_pairs"] == 0
    assert np.allclose(out["fb"], np.array([0.2, 0.4, 0.6], np.float32)[:, None, None])


def test_image_finite_and_binning_consistent():
    sc = S.make_scene(2000, seed=2)
    cam = S.make_camera(40, 32)
    out = O.vr_forward(sc, cam, want_list=True)
    fb = out["fb"]
    assert np.isfinite(fb).all() and fb.min() >= 0.0 and fb.max() > 0.05
    P = out["n_pairs"]
    assert P == int(out["point_offsets"][-1]) == len(out["point_list"])
    r = out["i_ranges"]
    assert (r[:, 1] >= r[:, 0]).all() and r[:, 1].max() == P
