"""Batched multi-view rendering: every view of a batch equals the same view
rendered alone (bit-exact images, point counts), per-scene gradients equal the
sum of the single-view gradients, and a captured CUDA graph replays to the
same results."""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import scene as S
from differentiable_gaussian_mixture_renderer_b200 import splat

pytestmark = pytest.mark.gpu

RES = [(64, 48), (96, 96), (83, 125), (128, 72), (48, 64)]  # 83 x 125: partial blend blocks at the edges


def _setup(cuda):
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene
    dev = torch.device("cuda:0")
    scenes = {"a": GaussianScene.from_numpy(S.make_scene(2000, seed=3), dev),
              "b": GaussianScene.from_numpy(S.make_scene(5000, seed=4, extent=1.5), dev)}
    views = []
    for k, (w, h) in enumerate(RES):
        cam = S.random_cameras(1, w, h, seed=10 + k)[0]
        views.append(("a" if k % 2 == 0 else "b", cam))
    return BatchRenderer(scenes, dev), scenes, views


def _single(scene, cam):
    return splat.splat_forward(scene.shs, scene.weights, scene.centroids, scene.scales, scene.rotations, cam.view,
                               cam.proj, cam.campos, (0.0, 0.0, 0.0), cam.width, cam.height, cam.tan_fovx,
                               cam.tan_fovy, scene.sh_degree)


def test_batch_forward_equals_single_views(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views)
    r.forward(p)
    torch.cuda.synchronize()
    assert not p.overflowed()
    total = 0
    for k, (sid, cam) in enumerate(views):
        fb, frame = _single(scenes[sid], cam)
        total += int(frame.stats[0].item())
        assert torch.equal(p.framebuffers[k], fb), f"view {k}"
    assert p.n_pairs() == total


def test_batch_backward_sums_single_view_gradients(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views, backward=True)
    gen = torch.Generator(device="cuda").manual_seed(2)
    for g in p.grad_framebuffers:
        g.copy_(torch.randn(g.shape, device="cuda", generator=gen))
    r.forward(p)
    r.backward(p)
    torch.cuda.synchronize()
    for sid, sc in scenes.items():
        want = None
        for k, (vsid, cam) in enumerate(views):
            if vsid != sid:
                continue
            fb, frame = _single(sc, cam)
            g = splat.splat_backward(frame, p.grad_framebuffers[k], sc.shs, sc.weights, sc.centroids, sc.scales,
                                     sc.rotations)
            want = list(g) if want is None else [a + b for a, b in zip(want, g)]
        got = p.grads[sid]
        for name, a, b in zip(("sh", "weights", "centroids", "scales", "rotations"), got, want):
            b = b.reshape(a.shape)
            scale = float(b.abs().max()) + 1e-12
            err = float((a - b).abs().max()) / scale
            assert err < 1e-4, f"scene {sid} grad {name}: rel err {err}"


def test_batch_graph_replay_matches_eager(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views, backward=True)
    for g in p.grad_framebuffers:
        g.fill_(0.5)
    r.forward(p)
    r.backward(p)
    torch.cuda.synchronize()
    eager = [fb.clone() for fb in p.framebuffers]
    eager_g = {k: [t.clone() for t in v] for k, v in p.grads.items()}
    for fb in p.framebuffers:
        fb.zero_()
    r.capture(p, backward=True)
    for _ in range(2):
        r.replay(p)
    torch.cuda.synchronize()
    for a, b in zip(p.framebuffers, eager):
        assert torch.equal(a, b)
    for k in eager_g:
        for a, b in zip(p.grads[k], eager_g[k]):
            # the per-pixel gradient sums use atomics: equal up to their order
            assert float((a - b).abs().max()) <= 1e-4 * float(b.abs().max()) + 1e-7


def test_batch_capacity_overflow_is_flagged(cuda):
    r, scenes, views = _setup(cuda)
    p = r.plan(views, capacity=100)
    r.forward(p)
    torch.cuda.synchronize()
    assert p.overflowed()
    assert p.n_pairs() > 100


def test_autotune_picks_a_depth_and_a_blend_block(cuda):
    from differentiable_gaussian_mixture_renderer_b200.batch import autotune
    r, scenes, views = _setup(cuda)
    best, timings = autotune(r, views, depths=(1, 2, 5), reps=1)
    assert set(timings) == {(d, b) for d in (1, 2, 5) for b in (8, 16)}
    assert best in timings and r.blend_block == best[1] and timings[best] == min(timings.values())
    assert all(t > 0 for t in timings.values())
    # with the backward, and the images of the picked setting still those of single views
    best, timings = autotune(r, views, depths=(2, 5), backward=True, reps=1)
    assert set(timings) == {(d, b) for d in (2, 5) for b in (8, 16)}
    p = r.plan(views)
    r.forward(p)
    torch.cuda.synchronize()
    for (sid, cam), fb in zip(views, p.framebuffers):
        want, _ = _single(scenes[sid], cam)
        assert torch.equal(fb, want)


@pytest.mark.gpu
@pytest.mark.parametrize("backward", [False, True])
def test_blend_block_sides_give_the_same_bits(cuda, backward):
    """The blend's 8x8 and 16x16 pixel blocks (the autotuner's block knob) walk
    the same tile lists: images, transmittance-derived contributor counts and
    point lists are the same bits; gradients agree up to the order of the
    per-pixel atomics."""
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer
    r, scenes, views = _setup(cuda)
    out = {}
    for blk in (8, 16):
        rb = BatchRenderer(scenes, cuda, blend_block=blk)
        p = rb.plan(views, backward=backward)
        if backward:
            gen = torch.Generator(device=cuda).manual_seed(4)
            for g in p.grad_framebuffers:
                g.copy_(torch.randn(g.shape, generator=gen, device=cuda))
        rb.forward(p)
        if backward:
            rb.backward(p)
        torch.cuda.synchronize()
        out[blk] = ([fb.clone() for fb in p.framebuffers], {k: [t.clone() for t in v] for k, v in p.grads.items()})
    for a, b in zip(out[8][0], out[16][0]):
        assert torch.equal(a, b)
    for sid in out[8][1]:
        for a, b in zip(out[8][1][sid], out[16][1][sid]):
            scale = float(b.abs().max()) + 1e-30
            assert float((a - b).abs().max()) <= 1e-5 * scale


def test_blend_block_must_be_8_or_16(cuda):
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer
    with pytest.raises(ValueError):
        BatchRenderer({}, cuda, blend_block=32)
