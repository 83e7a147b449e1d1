"""Batched volume marching (dgmr_vm_batch_*): every view of a batch equals the
same view marched alone through the reference-facing binding (bit-exact
images; the batch's pair count is the sum of the views'), per-scene
gradients equal the sum over the scene's views of the single-view gradients,
views without an image gradient take no part, and a captured CUDA graph
replays to the same results."""
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import cpp_binding, scene as S

from test_gpu_parity import cam_tensors

pytestmark = pytest.mark.gpu

RES = [(64, 48), (48, 64), (80, 56), (40, 40), (72, 24)]
NAMES = ("sh", "weights", "centroids", "scales", "rotations")
# the per-Gaussian totals are double sums whose order varies from run to run
GRAD_REL = 1e-5


def _setup(cuda):
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene
    scenes = {"a": GaussianScene.from_numpy(S.make_scene(1500, seed=3, sh_degree=1), cuda),
              "b": GaussianScene.from_numpy(S.make_scene(2500, seed=4, extent=1.5), cuda)}
    views = [("a" if k % 2 == 0 else "b", S.random_cameras(1, w, h, seed=20 + k)[0]) for k, (w, h) in enumerate(RES)]
    return BatchRenderer(scenes, cuda, kind="march"), scenes, views


def _args(sc, cam, cuda):
    view, proj, campos, bgt = cam_tensors(cam, cuda)
    return (sc.shs, sc.weights.reshape(-1, 1), sc.centroids, sc.scales, sc.rotations, view, proj, campos, bgt,
            cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, sc.sh_degree)


def _close(name, got, want):
    got, want = got.reshape(-1).double(), want.reshape(-1).double()
    scale = float(want.abs().max()) if want.numel() else 0.0
    err = float((got - want).abs().max()) if want.numel() else 0.0
    assert err <= GRAD_REL * max(scale, 1e-30), (name, err, scale)


def test_batch_march_forward_equals_single_views(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views)
    r.forward(p)
    torch.cuda.synchronize()
    assert not p.overflowed()
    total = 0
    for k, (sid, cam) in enumerate(views):
        cache = cpp_binding.forward(*_args(scenes[sid], cam, cuda))
        total += cache[11].numel()
        assert torch.equal(p.framebuffers[k], cache[0]), f"view {k}"
    assert p.n_pairs() == total


def test_batch_march_backward_sums_single_view_gradients(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views, backward=True)
    gen = torch.Generator(device="cuda").manual_seed(5)
    for g in p.grad_framebuffers:
        g.copy_(torch.randn(g.shape, device="cuda", generator=gen))
    r.forward(p)
    r.backward(p)
    torch.cuda.synchronize()
    assert int(p.stats[1].item()) == 0  # no flag raised (overflow, bounds, step limit)
    for sid, sc in scenes.items():
        want = None
        for k, (vid, cam) in enumerate(views):
            if vid != sid:
                continue
            args = _args(sc, cam, cuda)
            cache = cpp_binding.forward(*args)
            g = cpp_binding.backward(*args, p.grad_framebuffers[k], cache)
            want = list(g) if want is None else [a + b for a, b in zip(want, g)]
        for name, got, w in zip(NAMES, p.grads[sid], want):
            _close(f"{sid}.{name}", got, w)


def test_batch_march_views_without_gradient_take_no_part(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views, backward=True)
    gen = torch.Generator(device="cuda").manual_seed(6)
    for g in p.grad_framebuffers:
        g.copy_(torch.randn(g.shape, device="cuda", generator=gen))
    p.c_views[0].grad_framebuffer = None  # scene "a" keeps views 2 and 4
    r.forward(p)
    r.backward(p)
    torch.cuda.synchronize()
    sc = scenes["a"]
    want = None
    for k in (2, 4):
        args = _args(sc, views[k][1], cuda)
        cache = cpp_binding.forward(*args)
        g = cpp_binding.backward(*args, p.grad_framebuffers[k], cache)
        want = list(g) if want is None else [a + b for a, b in zip(want, g)]
    for name, got, w in zip(NAMES, p.grads["a"], want):
        _close(f"a.{name}", got, w)


def test_batch_march_graph_replay(cuda):
    r, scenes, views = _setup(cuda)
    p = r.capture(r.plan(views, backward=True), backward=True)
    for g in p.grad_framebuffers:
        g.fill_(0.5)
    r.replay(p)
    torch.cuda.synchronize()
    first = [fb.clone() for fb in p.framebuffers]
    grads = [t.clone() for t in p.grads["b"]]
    for fb in p.framebuffers:
        fb.zero_()
    r.replay(p)
    torch.cuda.synchronize()
    for a, b in zip(first, p.framebuffers):
        assert torch.equal(a, b)
    for name, a, b in zip(NAMES, grads, p.grads["b"]):
        _close(f"replay.{name}", b, a)
    sid, cam = views[1]
    assert torch.equal(first[1], cpp_binding.forward(*_args(scenes[sid], cam, cuda))[0])


def test_batch_march_autotune_picks_a_depth(cuda):
    """The native autotuner (dgmr_batch_autotune) on marcher batches, forward
    and backward: one time per depth (no blend block: 0), the best among them,
    and the renders afterwards still equal the single views."""
    from differentiable_gaussian_mixture_renderer_b200.batch import autotune
    r, scenes, views = _setup(cuda)
    (depth, block), timings = autotune(r, views, depths=(1, 2, 5), backward=True, reps=1)
    assert set(timings) == {(1, 0), (2, 0), (5, 0)} and block == 0
    assert timings[(depth, 0)] == min(timings.values()) and all(t > 0 for t in timings.values())
    p = r.plan(views)
    r.forward(p)
    for (sid, cam), fb in zip(views, p.framebuffers):
        want = cpp_binding.forward(*_args(scenes[sid], cam, cuda))[0]
        assert torch.equal(fb, want)
