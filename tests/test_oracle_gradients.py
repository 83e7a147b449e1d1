"""Finite-difference checks of the oracle's adjoints (float64, CPU).

The reference checks every adjoint of its device math by central differences
(unittests/grad_math.cu, unittests/grad_inria_splatter_render.cu); here the
whole pipelines are checked the same way: a random upstream image gradient G,
loss = sum(render * G), 25 random parameters per input tensor, eps 1e-6
(1e-7 where 1e-6 straddles a discrete decision).
The volume marcher runs with fixed sample sections (the reference's
DGMR_TORCH_GRAD_CHECK_CONST_SAMPLES mode), because adaptive sampling makes the
forward piecewise constant in the sample positions.
"""
import numpy as np
import pytest

from differentiable_gaussian_mixture_renderer_b200 import scene as S
from oracle import oracle as O

TOL = 1e-3


def as_f64(sc):
    for k in ("centroids", "sh", "weights", "scales", "rotations"):
        setattr(sc, k, getattr(sc, k).astype(np.float64))
    return sc


def fd_check(sc, grads, loss, rng, per_tensor=25, eps=1e-6):
    bad = []
    for name in ("centroids", "scales", "rotations", "weights", "sh"):
        flat = getattr(sc, name).reshape(-1)
        ga = grads[name].reshape(-1)
        for i in rng.choice(flat.size, size=min(per_tensor, flat.size), replace=False):
            o = flat[i]
            for e in (eps, eps / 10):
                # a discrete decision of the renderer (a depth order, a rect edge, a
                # skipped sample) within e of the parameter adds jump / 2e to the
                # difference quotient; a tenth of the step no longer straddles it,
                # while a wrong adjoint disagrees at both steps
                flat[i] = o + e
                lp = loss()
                flat[i] = o - e
                lm = loss()
                flat[i] = o
                fd = (lp - lm) / (2 * e)
                err = abs(fd - ga[i]) / max(1e-4, abs(fd), abs(ga[i]))
                if err <= TOL:
                    break
            else:
                bad.append((name, int(i), fd, float(ga[i]), err))
    return bad


FORMULATIONS = [None, "opacity", "mass", "density", "ots", "ols"]


@pytest.mark.parametrize("formulation", FORMULATIONS)
def test_splat_backward_matches_finite_differences(formulation):
    """Every formulation of math.h:322-380 (None = the splat default, Ots);
    the reference checks each one's splat adjoint the same way
    (unittests/grad_math.cu:435-455)."""
    sc = as_f64(S.make_scene(60, seed=3, sh_degree=3, scale_range=(0.05, 0.3)))
    sc.formulation = formulation
    cam = S.make_camera(48, 40, eye=(0.3, -0.2, -3.0), dtype=np.float64)
    rng = np.random.default_rng(2)
    G = rng.normal(size=(3, 40, 48))
    bg = np.array([0.1, 0.2, 0.3])
    _, g = O.splat_render_f64(sc, cam, grad_fb=G, bg=bg)
    loss = lambda: float((O.splat_render_f64(sc, cam, bg=bg) * G).sum())
    bad = fd_check(sc, g, loss, rng)
    assert not bad, bad


@pytest.mark.parametrize("seed,formulation", [(5, None), (9, None), (5, "mass"), (5, "density"), (9, "ots"),
                                              (9, "ols")])
def test_vol_marcher_backward_matches_finite_differences(seed, formulation):
    """None = the marcher default (Opacity); the others exercise the
    weight_to_mass adjoint of each formulation (grad/math.h:284-330)."""
    sc = as_f64(S.make_scene(40, seed=seed, sh_degree=2, scale_range=(0.05, 0.25), extent=0.6))
    sc.formulation = formulation
    cam = S.make_camera(24, 20, eye=(0.2, -0.1, -3.0), dtype=np.float64)
    O.set_const_samples([(2.0, 3.0, 1.0 / 31), (3.0, 4.0, 1.0 / 31)])
    try:
        rng = np.random.default_rng(seed)
        G = rng.normal(size=(3, 20, 24))
        bg = np.array([0.1, 0.2, 0.3])
        c = O.vm_forward(sc, cam, bg=bg, dtype=np.float64)
        assert c["remaining_transparency"].min() < 0.9  # the scene does occlude
        g = O.vm_backward(sc, cam, c, G, bg=bg, dtype=np.float64)
        loss = lambda: float((O.vm_forward(sc, cam, bg=bg, dtype=np.float64)["fb"] * G).sum())
        bad = fd_check(sc, g, loss, rng)
        assert not bad, bad
    finally:
        O.set_const_samples([])


def test_c1_scene_backward_matches_finite_differences():
    """The splat configuration c1 (200,000 Gaussians, means in [-2, 2]^3,
    camera at distance 3) seen through a 64x64 window at the centre of its
    1024x1024 frame (same rays, 1/16 of the field of view): 64 parameters of
    Gaussians that reach the window, central differences in float64.
    eps is 1e-6, not 1e-3: this renderer's hard decisions -- depth-order swaps
    of overlapping splats, the alpha >= 1/255 cutoff, saturation -- put jumps
    into a 1e-3 difference quotient (measured on the full 1024^2 float32 frame:
    11 of 17 parameters with a non-zero gradient off by 25-170 %, the smooth
    ones -- colours, a large scale gradient -- within 2-4 %)."""
    import math
    sc = as_f64(S.make_scene(200_000, seed=0, extent=2.0))
    cam = S.make_camera(64, 64, fovy_deg=2.0 * math.degrees(math.atan(math.tan(math.radians(30.0)) / 16.0)),
                        dtype=np.float64)
    rng = np.random.default_rng(3)
    G = rng.normal(size=(3, 64, 64))
    _, g = O.splat_render_f64(sc, cam, grad_fb=G)
    loss = lambda: float((O.splat_render_f64(sc, cam) * G).sum())
    live = np.nonzero(np.abs(g["centroids"]).sum(axis=1) > 0)[0]
    assert live.size >= 64
    # 64 parameters: every tensor of 64 random live Gaussians, in turn
    picks = rng.choice(live, size=64, replace=False)
    bad = []
    for k, i in enumerate(picks):
        name = ("centroids", "scales", "rotations", "weights", "sh")[k % 5]
        flat = getattr(sc, name).reshape(sc.n, -1)
        ga = g[name].reshape(sc.n, -1)
        j = int(rng.integers(flat.shape[1] if name != "sh" else 3))
        o = flat[i, j]
        for e in (1e-6, 1e-7):
            flat[i, j] = o + e
            lp = loss()
            flat[i, j] = o - e
            lm = loss()
            flat[i, j] = o
            fd = (lp - lm) / (2 * e)
            err = abs(fd - ga[i, j]) / max(1e-4, abs(fd), abs(ga[i, j]))
            if err <= TOL:
                break
        else:
            bad.append((name, int(i), j, fd, float(ga[i, j]), err))
    assert not bad, bad
