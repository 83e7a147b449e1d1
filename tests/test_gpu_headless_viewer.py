"""The headless viewer (C++ over include/dgmr_b200_sibr.hpp, the reference's
sibr_interfaces without a window) renders the same frames as the Python API:
bit-identical framebuffers for the splat, the marcher and vol_raster, and the
PPM is the framebuffer's 8-bit conversion."""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import build, cpp_binding, headless, scene as S, splat, vol_raster

pytestmark = pytest.mark.gpu

BG = (0.1, 0.2, 0.3)


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    build.build_viewer()
    d = tmp_path_factory.mktemp("viewer")
    sc = S.make_scene(6000, seed=21, sh_degree=1)
    cam = S.make_camera(120, 88, eye=(0.3, -0.4, -3.0))
    headless.write_scene(str(d / "s.bin"), sc)
    headless.write_camera(str(d / "c.bin"), cam)
    return d, sc, cam


def _tensors(sc, cam, dev):
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    return (t(sc.sh), t(sc.weights).reshape(-1, 1), t(sc.centroids), t(sc.scales), t(sc.rotations), t(cam.view),
            t(cam.proj), t(cam.campos), t(np.array(BG, np.float32)))


def _python_frame(renderer, sc, cam, dev, **kw):
    shs, w, mu, s, q, view, proj, campos, bg = _tensors(sc, cam, dev)
    args = (shs, w, mu, s, q, view, proj, campos, bg, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, sc.sh_degree)
    if renderer == "splat":
        fb, _ = splat.splat_forward(*args, formulation=kw.get("formulation"))
        return fb
    if renderer == "march":
        return cpp_binding.forward(*args, render_mode=kw.get("mode", "full"), formulation=kw.get("formulation"))[0]
    return vol_raster.forward(*args, render_mode=kw.get("mode", "full"), formulation=kw.get("formulation"))


@pytest.mark.parametrize("renderer,kw", [("splat", {}), ("march", {}), ("raster", {}), ("splat", {"formulation": "mass"}),
                                         ("march", {"mode": "depth"}), ("raster", {"formulation": "opacity"})])
def test_viewer_frame_equals_python_api(cuda, files, renderer, kw):
    d, sc, cam = files
    raw, ppm = str(d / f"{renderer}.f32"), str(d / f"{renderer}.ppm")
    rep = headless.run(str(d / "s.bin"), str(d / "c.bin"), renderer, frames=3, raw=raw, ppm=ppm, background=BG, **kw)
    assert rep["width"] == cam.width and rep["height"] == cam.height and rep["flags"] == 0 and rep["n_pairs"] > 0
    assert rep["ms_per_frame"] > 0
    got = headless.read_raw(raw, cam.width, cam.height)
    want = _python_frame(renderer, sc, cam, cuda, **kw).cpu().numpy()
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(headless.read_ppm(ppm), headless.to_ppm_bytes(got))
