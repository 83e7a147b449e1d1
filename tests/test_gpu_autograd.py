"""The autograd wrappers on the GPU: vol_marcher.apply (drop-in for
python_bindings/vol_marcher.py) and splat.render.

* torch.autograd.gradcheck of vol_marcher.apply in float64 with fixed sample
  sections (the reference's DGMR_TORCH_GRAD_CHECK_CONST_SAMPLES mode);
* loss.backward() through both ops gives the oracle's gradients (1e-3).
"""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import cpp_binding, scene as S, splat, vol_marcher
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def tensors(sc, dev, dtype, grad=True):
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=dev, requires_grad=grad)
    return t(sc.sh), t(sc.weights.reshape(-1, 1)), t(sc.centroids), t(sc.scales), t(sc.rotations)


def test_vol_marcher_gradcheck_const_samples(cuda):
    sc = S.make_scene(6, seed=5, sh_degree=1, scale_range=(0.15, 0.3), extent=0.3)
    cam = S.make_camera(16, 16, eye=(0.05, -0.05, -3.0), dtype=np.float64)
    view, proj, campos = (torch.tensor(a, dtype=torch.float64, device=cuda) for a in (cam.view, cam.proj, cam.campos))
    bg = torch.tensor([0.1, 0.2, 0.3], dtype=torch.float64, device=cuda)
    inputs = tensors(sc, cuda, torch.float64)
    cpp_binding.set_const_samples([(2.0, 3.0, 1.0 / 31), (3.0, 4.0, 1.0 / 31)])
    try:
        f = lambda *x: vol_marcher.apply(*x, view, proj, campos, bg, 16, 16, cam.tan_fovx, cam.tan_fovy, 1)
        assert f(*inputs).min() < 0.5  # something is in view
        assert torch.autograd.gradcheck(f, inputs, eps=1e-6, atol=1e-5, rtol=1e-3, nondet_tol=1e-9)
    finally:
        cpp_binding.set_const_samples([])


def test_vol_marcher_apply_backward_matches_oracle(cuda):
    sc = S.make_scene(1200, seed=7, sh_degree=1)
    cam = S.make_camera(40, 32, eye=(0.2, 0.1, -3.0))
    view, proj, campos = (torch.tensor(a, device=cuda) for a in (cam.view, cam.proj, cam.campos))
    bg = torch.tensor([0.2, 0.3, 0.1], device=cuda)
    ins = tensors(sc, cuda, torch.float32)
    G = np.random.default_rng(3).normal(size=(3, cam.height, cam.width)).astype(np.float32)
    img = vol_marcher.apply(*ins, view, proj, campos, bg, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, 1)
    (img * torch.tensor(G, device=cuda)).sum().backward()
    ref = O.vm_forward(sc, cam, bg=np.array([0.2, 0.3, 0.1], np.float32))
    assert np.abs(img.detach().cpu().numpy() - ref["fb"]).max() <= 1e-4
    g = O.vm_backward(sc, cam, ref, G, bg=np.array([0.2, 0.3, 0.1], np.float32))
    for t, name in zip(ins, ("sh", "weights", "centroids", "scales", "rotations")):
        a = t.grad.cpu().numpy().reshape(g[name].shape)
        b = g[name]
        assert np.max(np.abs(a - b) / (np.abs(b) + 1e-3 * np.abs(b).max())) <= 1e-3, name


def test_splat_render_backward_matches_oracle(cuda):
    sc = S.make_scene(3000, seed=8, sh_degree=2)
    cam = S.make_camera(96, 72, eye=(-0.3, 0.2, -3.0))
    view, proj, campos = (torch.tensor(a, device=cuda) for a in (cam.view, cam.proj, cam.campos))
    bg = torch.tensor([0.0, 0.1, 0.2], device=cuda)
    ins = tensors(sc, cuda, torch.float32)
    G = np.random.default_rng(4).normal(size=(3, cam.height, cam.width)).astype(np.float32)
    img = splat.render(*ins, view, proj, campos, bg, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, 2)
    (img * torch.tensor(G, device=cuda)).sum().backward()
    bgn = np.array([0.0, 0.1, 0.2], np.float32)
    ref = O.splat_forward(sc, cam, bg=bgn)
    assert np.abs(img.detach().cpu().numpy() - ref["fb"]).max() <= 1e-4
    g = O.splat_backward(sc, cam, ref, G, bg=bgn)
    for t, name in zip(ins, ("sh", "weights", "centroids", "scales", "rotations")):
        a = t.grad.cpu().numpy().reshape(g[name].shape)
        b = g[name]
        assert np.max(np.abs(a - b) / (np.abs(b) + 1e-3 * np.abs(b).max())) <= 1e-3, name
