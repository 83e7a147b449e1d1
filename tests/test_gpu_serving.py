"""Continuous batching: every request's result is the same served alone and in
the mix (images bit-identical, gradients equal up to the order of the
per-pixel atomics), with batches that mix scenes, resolutions and gradient
requests, under a tight HBM budget too."""
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import scene as S
from differentiable_gaussian_mixture_renderer_b200 import splat

pytestmark = pytest.mark.gpu

RES = [(64, 64), (96, 64), (128, 96), (80, 48)]


def _scenes(dev):
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene
    return {"a": GaussianScene.from_numpy(S.make_scene(1500, seed=5), dev),
            "b": GaussianScene.from_numpy(S.make_scene(4000, seed=6), dev),
            "c": GaussianScene.from_numpy(S.make_scene(2500, seed=7, extent=1.5), dev)}


def _requests(dev, n=20):
    from differentiable_gaussian_mixture_renderer_b200.serving import ServeRequest
    gen = torch.Generator(device=dev).manual_seed(9)
    reqs = []
    for k in range(n):
        w, h = RES[k % len(RES)]
        cam = S.random_cameras(1, w, h, seed=200 + k)[0]
        bwd = k % 4 == 1
        g = torch.randn((3, h, w), device=dev, generator=gen) if bwd else None
        reqs.append(ServeRequest("abc"[k % 3], cam, backward=bwd, grad_image=g))
    return reqs


def _alone(scene, req):
    cam = req.camera
    fb, frame = splat.splat_forward(scene.shs, scene.weights, scene.centroids, scene.scales, scene.rotations, cam.view,
                                    cam.proj, cam.campos, (0.0, 0.0, 0.0), cam.width, cam.height, cam.tan_fovx,
                                    cam.tan_fovy, scene.sh_degree)
    grads = None
    if req.backward:
        grads = splat.splat_backward(frame, req.grad_image, scene.shs, scene.weights, scene.centroids, scene.scales,
                                     scene.rotations)
    return fb, grads


def _check(scenes, reqs):
    for k, req in enumerate(reqs):
        fb, grads = _alone(scenes[req.scene_id], req)
        assert torch.equal(req.image, fb), f"request {k}: image differs from the request served alone"
        if req.backward:
            for name, a, b in zip(("sh", "weights", "centroids", "scales", "rotations"), req.grads, grads):
                b = b.reshape(a.shape)
                err = float((a - b).abs().max()) / (float(b.abs().max()) + 1e-12)
                assert err < 1e-4, f"request {k}: grad {name} rel err {err}"


@pytest.mark.parametrize("n_slots,max_batch", [(3, 4), (2, 8)])
def test_results_equal_alone_and_in_the_mix(cuda, n_slots, max_batch):
    from differentiable_gaussian_mixture_renderer_b200.serving import ContinuousServer
    dev = torch.device("cuda:0")
    scenes = _scenes(dev)
    server = ContinuousServer(scenes, dev, n_slots=n_slots, max_batch=max_batch)
    reqs = _requests(dev)
    for r in reqs[:7]:
        server.submit(r)
    server.poll()  # first batches go out while the rest arrive
    for r in reqs[7:]:
        server.submit(r)
        server.poll()
    server.drain()
    torch.cuda.synchronize()
    assert len(server.completed) == len(reqs)
    assert max(r.batch_size for r in reqs) > 1  # requests were actually mixed
    assert any(r.backward and r.batch_size > 1 for r in reqs)
    _check(scenes, reqs)
    assert server.budget.in_use == 0


def test_tight_hbm_budget_defers_requests(cuda):
    from differentiable_gaussian_mixture_renderer_b200.serving import ContinuousServer
    dev = torch.device("cuda:0")
    scenes = _scenes(dev)
    reqs = _requests(dev, n=8)
    probe = ContinuousServer(scenes, dev)
    one = max(probe._cost([r]) for r in reqs)
    server = ContinuousServer(scenes, dev, n_slots=3, max_batch=8, hbm_budget_bytes=int(one * 1.2))
    for r in reqs:
        server.submit(r)
    server.drain()
    torch.cuda.synchronize()
    assert len(server.completed) == len(reqs)
    assert server.budget.peak <= server.budget.budget
    assert server.deferred > 0  # requests waited for memory instead of over-committing it
    _check(scenes, reqs)


def test_overflowing_capacity_is_rerendered(cuda):
    from differentiable_gaussian_mixture_renderer_b200.serving import ContinuousServer
    dev = torch.device("cuda:0")
    scenes = _scenes(dev)
    reqs = _requests(dev, n=6)
    server = ContinuousServer(scenes, dev, n_slots=2, max_batch=3)
    for r in reqs:  # learnt capacities far too small
        server.capacity[(r.scene_id, r.camera.width, r.camera.height)] = 16
    for r in reqs:
        server.submit(r)
    server.drain()
    torch.cuda.synchronize()
    assert server.rerenders > 0 and all(r.rerendered for r in reqs)
    _check(scenes, reqs)


@pytest.mark.parametrize("to_host", [False, True])
def test_render_server_results_are_not_reused(cuda, to_host):
    """RenderServer: 8 results kept from 4 slots -- each still equals its frame
    rendered alone after later requests reused the slots; released buffers are
    handed to later requests instead of new ones."""
    from differentiable_gaussian_mixture_renderer_b200.serving import RenderServer, Request
    scenes = _scenes(cuda)
    server = RenderServer(scenes, cuda, n_slots=4)
    reqs = []
    for k in range(8):
        w, h = RES[k % 2]
        reqs.append(server.submit(Request("ab"[k % 2], S.random_cameras(1, w, h, seed=300 + k)[0], to_host=to_host)))
    server.drain()
    for k, req in enumerate(reqs):
        fb = _render_alone(scenes[req.scene_id], req.camera)
        assert req.image.is_pinned() if to_host else req.image.is_cuda
        img = req.image.to(cuda) if to_host else req.image
        assert torch.equal(img, fb), f"request {k}: image was overwritten by a later request"
    held = {r.image.data_ptr() for r in reqs}  # eight distinct result buffers
    assert len(held) == 8
    for r in reqs:
        r.release()
        assert r.image is None
    again = server.submit(Request("a", S.random_cameras(1, *RES[0], seed=400)[0], to_host=to_host))
    server.drain()
    assert again.image.data_ptr() in held
    fb = _render_alone(scenes["a"], again.camera)
    assert torch.equal(again.image.to(cuda) if to_host else again.image, fb)


@pytest.mark.parametrize("to_host", [False, True])
def test_render_server_rerenders_overflowed_frames(cuda, to_host):
    """RenderServer with learnt capacities far too small: the frames launched
    with them overflow, render again exactly sized before they complete, and
    every result equals its frame rendered alone (a grown capacity serves the
    requests launched after it)."""
    from differentiable_gaussian_mixture_renderer_b200.serving import RenderServer, Request
    scenes = _scenes(cuda)
    server = RenderServer(scenes, cuda, n_slots=3)
    reqs = [Request("ab"[k % 2], S.random_cameras(1, *RES[k % 2], seed=500 + k)[0], to_host=to_host) for k in range(9)]
    for r in reqs:
        server.capacity[(r.scene_id, r.camera.width, r.camera.height)] = 16
    for r in reqs:
        server.submit(r)
    server.drain()
    assert reqs[0].rerendered and server.rerenders >= 2  # the first frame of each key at least
    assert len(server.completed) == len(reqs)
    for k, req in enumerate(reqs):
        fb = _render_alone(scenes[req.scene_id], req.camera)
        assert torch.equal(req.image.to(cuda) if to_host else req.image, fb), f"request {k}"
        assert req.meta["n_pairs"] > 16


def _render_alone(scene, cam):
    fb, _ = splat.splat_forward(scene.shs, scene.weights, scene.centroids, scene.scales, scene.rotations, cam.view,
                                cam.proj, cam.campos, (0.0, 0.0, 0.0), cam.width, cam.height, cam.tan_fovx,
                                cam.tan_fovy, scene.sh_degree)
    return fb
