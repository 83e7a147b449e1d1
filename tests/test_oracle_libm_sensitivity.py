"""What sharing exp / log / erf between the CUDA kernels and the oracle hides.

The kernels and the default oracle build use fixed-sequence float routines
that give the same bits (csrc/dgmr_fmath.h, and the oracle's own coding of
the same methods, oracle/dgmr_oracle_fmath.h), so GPU and oracle take every
threshold decision the same way.  The reference calls CUDA's expf / erff instead.  The oracle is
therefore also built with the host libm's expf / logf / erff (the nearest
stand-in available here), and these tests measure the difference:

* end to end: the two builds' outputs on the 10k / 256^2 splat frame and on a
  128^2 crop (same focal length, centre of the image) of the 100k / 512^2
  marcher frame -- rectangles, tile counts, point lists and contributor
  counts identical, images within the stated bounds;
* per decision: every float alpha >= 1/255 (splat), ray-section mass >= 1/255
  (marcher) and isoline-radius ceil (marcher rectangle) decision taken with
  both functions on the same argument: none flips, and the decisions within
  16 float ulps of their threshold -- the only ones any exp / log within 16
  ulps of the fixed-sequence routines could flip -- are a few per ten million.
Measured when written: splat image 1.8e-7, marcher crop 5.8e-6; 4 of 13.6M
alpha decisions, 4 of 12.2M section-mass decisions and 4 of 200k radii near
their thresholds, no flips.
"""
import math

import numpy as np

from differentiable_gaussian_mixture_renderer_b200 import scene as S
from oracle import oracle as O


def test_splat_c0_libm_build_and_decisions():
    sc = S.make_scene(10_000, seed=0)
    cam = S.make_camera(256, 256)
    with O.decision_audit() as audit:
        a = O.splat_forward(sc, cam)
    with O.libm_transcendentals():
        b = O.splat_forward(sc, cam)
    assert a["n_pairs"] == b["n_pairs"]
    for k in ("rects", "tiles_touched", "point_offsets", "i_ranges", "point_list", "keys", "n_contrib"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert float(np.abs(a["fb"] - b["fb"]).max()) <= 1e-6
    seen, flipped, near = audit["alpha"]
    assert seen > 10_000_000 and flipped == 0
    assert near <= 1e-6 * seen, audit


def test_vol_marcher_c2_crop_libm_build_and_decisions():
    sc = S.make_scene(100_000, seed=0)
    fovy = math.degrees(2.0 * math.atan(math.tan(math.radians(30.0)) / 4.0))
    cam = S.make_camera(128, 128, fovy_deg=fovy)
    with O.decision_audit() as audit:
        a = O.vm_forward(sc, cam)
    with O.libm_transcendentals():
        b = O.vm_forward(sc, cam)
    for k in ("rects", "tiles_touched", "point_offsets", "i_ranges", "b_point_list"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert float(np.abs(a["fb"] - b["fb"]).max()) <= 1e-4
    assert float(np.abs(a["remaining_transparency"] - b["remaining_transparency"]).max()) <= 1e-4
    for kind in ("section_mass", "rect"):
        seen, flipped, near = audit[kind]
        assert seen > 0 and flipped == 0, (kind, audit)
    seen, _, near = audit["section_mass"]
    assert seen > 10_000_000 and near <= 1e-6 * seen, audit
    seen, _, near = audit["rect"]
    assert near <= 1e-4 * seen, audit
