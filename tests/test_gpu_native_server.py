"""The C++ continuous-batching server (dgmr_server_*, through NativeServer):
every request's result equals the plain call's -- splat requests against
splat_forward / splat_backward, vol_marcher requests against
cpp_binding.forward / backward -- alone and in a mix of scenes, resolutions,
renderers and gradient requests; also under a tight HBM budget (requests
wait instead of over-committing memory) and with pair capacities far too
small (batches render again, exactly sized)."""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import cpp_binding, scene as S
from test_gpu_serving import RES, _alone, _check, _requests, _scenes

pytestmark = pytest.mark.gpu


def _march_alone(scene, req):
    cam = req.camera
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device=scene.centroids.device)
    v, p, c = t(cam.view), t(cam.proj), t(cam.campos)
    bg = torch.zeros(3, device=scene.centroids.device)
    w = scene.weights.reshape(-1, 1)
    cache = cpp_binding.forward(scene.shs, w, scene.centroids, scene.scales, scene.rotations, v, p, c, bg, cam.width,
                                cam.height, cam.tan_fovx, cam.tan_fovy, scene.sh_degree)
    grads = None
    if req.backward:
        grads = cpp_binding.backward(scene.shs, w, scene.centroids, scene.scales, scene.rotations, v, p, c, bg,
                                     cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, scene.sh_degree,
                                     req.grad_image, cache)
    return cache[0], grads


def _check_all(scenes, reqs):
    splats = [r for r in reqs if r.kind == "splat"]
    _check(scenes, splats)
    for k, req in enumerate(r for r in reqs if r.kind == "march"):
        fb, grads = _march_alone(scenes[req.scene_id], req)
        assert torch.equal(req.image, fb), f"marcher request {k}: image differs from the request served alone"
        if req.backward:
            for name, a, b in zip(("sh", "weights", "centroids", "scales", "rotations"), req.grads, grads):
                b = b.reshape(a.shape)
                err = float((a - b).abs().max()) / (float(b.abs().max()) + 1e-12)
                assert err < 1e-4, f"marcher request {k}: grad {name} rel err {err}"


def _mixed(dev, n=20):
    reqs = _requests(dev, n)
    for k, r in enumerate(reqs):
        if k % 5 == 3:
            r.kind = "march"
    return reqs


@pytest.mark.parametrize("n_slots,max_batch", [(3, 4), (2, 8)])
def test_native_server_results_equal_alone_and_in_the_mix(cuda, n_slots, max_batch):
    from differentiable_gaussian_mixture_renderer_b200.serving import NativeServer
    scenes = _scenes(cuda)
    server = NativeServer(scenes, cuda, n_slots=n_slots, max_batch=max_batch)
    reqs = _mixed(cuda)
    for r in reqs[:7]:
        server.submit(r)
    server.poll()
    for r in reqs[7:]:
        server.submit(r)
        server.poll()
    server.drain()
    assert len(server.completed) == len(reqs)
    assert all(r.status == 0 for r in reqs)
    assert max(r.batch_size for r in reqs) > 1
    assert any(r.backward and r.kind == "splat" and r.batch_size > 1 for r in reqs)
    assert any(r.backward and r.kind == "march" for r in reqs)
    _check_all(scenes, reqs)
    st = server.stats()
    assert st["hbm_in_use_bytes"] == 0 and st["submitted"] == len(reqs)
    server.close()


def test_native_server_copies_to_pinned_host_images(cuda):
    from differentiable_gaussian_mixture_renderer_b200.serving import NativeServer, ServeRequest
    import time
    scenes = _scenes(cuda)
    server = NativeServer(scenes, cuda, n_slots=2, max_batch=4)
    t_before = time.perf_counter()
    reqs = []
    for k in range(6):
        w, h = RES[k % len(RES)]
        r = ServeRequest("ab"[k % 2], S.random_cameras(1, w, h, seed=500 + k)[0], kind="march" if k == 5 else "splat")
        r.host_image = torch.empty((3, h, w), dtype=torch.float32, pin_memory=True)
        reqs.append(server.submit(r))
    server.drain()
    t_after = time.perf_counter()
    for r in reqs:
        assert torch.equal(r.host_image, r.image.cpu())
        # completion times are on this process's clock: after submission, before drain returned
        assert t_before - 1e-3 <= r.t_launch <= r.t_done <= t_after + 1e-3, (t_before, r.t_launch, r.t_done, t_after)
    _check_all(scenes, reqs)
    server.close()


def test_native_server_tight_budget_defers(cuda):
    from differentiable_gaussian_mixture_renderer_b200.serving import ContinuousServer, NativeServer
    scenes = _scenes(cuda)
    reqs = _requests(cuda, n=8)
    probe = ContinuousServer(scenes, cuda)
    one = max(probe._cost([r]) for r in reqs)
    server = NativeServer(scenes, cuda, n_slots=3, max_batch=8, hbm_budget_bytes=int(one * 1.5))
    for r in reqs:
        server.submit(r)
    server.drain()
    st = server.stats()
    assert st["hbm_peak_bytes"] <= st["hbm_budget_bytes"]
    assert st["deferred"] > 0
    _check_all(scenes, reqs)
    server.close()


def test_native_server_rerenders_overflowed_batches(cuda):
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene, NativeServer, ServeRequest
    scenes = {"big": GaussianScene.from_numpy(S.make_scene(20000, seed=12), cuda)}
    # capacities at a quarter of the pairs seen: later frames of a key overflow and render again
    server = NativeServer(scenes, cuda, n_slots=2, max_batch=4, capacity_margin=0.25)
    gen = torch.Generator(device=cuda).manual_seed(4)
    reqs = []
    for k in range(8):
        cam = S.random_cameras(1, 256, 256, seed=700 + k)[0]
        bwd = k % 3 == 0
        g = torch.randn((3, 256, 256), device=cuda, generator=gen) if bwd else None
        reqs.append(server.submit(ServeRequest("big", cam, backward=bwd, grad_image=g,
                                               kind="march" if k == 4 else "splat")))
    server.drain()
    assert server.stats()["rerenders"] > 0 and any(r.rerendered for r in reqs)
    _check_all(scenes, reqs)
    server.close()


def test_native_server_capacity_grows_once_per_overflow(cuda):
    """A batch of many requests of one (scene, resolution) that overflows grows
    that key's capacity once, not once per request: memory held stays of the
    order of the frames' real needs."""
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene, NativeServer, ServeRequest
    scenes = {"big": GaussianScene.from_numpy(S.make_scene(20000, seed=12), cuda)}
    server = NativeServer(scenes, cuda, n_slots=2, max_batch=8, capacity_margin=0.25)
    reqs = [server.submit(ServeRequest("big", S.random_cameras(1, 256, 256, seed=900 + k)[0])) for k in range(32)]
    server.drain()
    st = server.stats()
    assert st["rerenders"] > 0
    assert st["hbm_peak_bytes"] < (1 << 30), st
    _check_all(scenes, reqs)
    server.close()


def test_native_server_pixel_cap_keeps_large_views_apart(cuda):
    """max_batch_pixels: a batch takes no further view once its pixels would
    pass the cap (it always takes one); small views still share batches."""
    from differentiable_gaussian_mixture_renderer_b200.serving import NativeServer, ServeRequest
    scenes = _scenes(cuda)
    server = NativeServer(scenes, cuda, n_slots=1, max_batch=8, max_batch_pixels=128 * 96)
    big = [ServeRequest("a", S.random_cameras(1, 128, 96, seed=800 + k)[0]) for k in range(4)]
    small = [ServeRequest("b", S.random_cameras(1, 32, 24, seed=850 + k)[0]) for k in range(8)]
    for r in big + small:
        server.submit(r)
    server.drain()
    assert all(r.batch_size == 1 for r in big)
    assert max(r.batch_size for r in small) > 1
    _check_all(scenes, big + small)
    server.close()


def test_native_server_batches_marcher_requests(cuda):
    """Marcher requests of small views share batches (dgmr_vm_batch_*), with
    and without gradients, across two scenes; a batch holds one kind, and
    every result equals the plain call's."""
    from differentiable_gaussian_mixture_renderer_b200.serving import NativeServer, ServeRequest
    scenes = _scenes(cuda)
    server = NativeServer(scenes, cuda, n_slots=1, max_batch=8)
    gen = torch.Generator(device=cuda).manual_seed(9)
    reqs = []
    for k in range(14):
        cam = S.random_cameras(1, 48, 40, seed=950 + k)[0]
        bwd = k % 3 == 1
        g = torch.randn((3, 40, 48), device=cuda, generator=gen) if bwd else None
        kind = "splat" if k == 6 else "march"
        reqs.append(ServeRequest("a" if k % 2 else "b", cam, backward=bwd, grad_image=g, kind=kind))
    for r in reqs:
        server.submit(r)
    server.drain()
    assert all(r.status == 0 for r in reqs)
    march = [r for r in reqs if r.kind == "march"]
    assert max(r.batch_size for r in march) > 1
    assert any(r.backward and r.batch_size > 1 for r in march)
    _check_all(scenes, reqs)
    server.close()
