"""Known-answer tests of the reference, run on the CPU.

* unittests/marching_steps.cpp -- DensityArray combine/put KATs (extracted to
  tests/golden/marching_steps_kats.json by tests/golden/extract_reference_kats.py),
  the srand(0) randomised invariant test and the sampler checks; each against
  the oracle AND the product's host/device section set (dgmr_sections.h).
* unittests/piecewise_linear.cpp -- FunctionGroup sample values, mass
  conservation of create_approximation, volume_integrate against a 1e6-step
  numeric integral within 1/256 (product header dgmr_volume_fit.h).
* unittests/raster_bin_sizer.cpp -- the RasterBinSizer property sections.
* unittests/math.cpp -- larger2 / smaller2 (the two largest / smallest scales,
  used by the Ots / Ols mass formulations).  Its other cases test
  rotation_matrix_from, orient_filter_kernel and
  gaussian_to_point_distance_bounds, which nothing on the rendering path calls.

The elementary functions are pinned here too: the oracle's own exp / log / erf
(oracle/dgmr_oracle_fmath.h) and the CUDA library's (csrc/dgmr_fmath.h) are
separate codings of the same published methods and must agree bit for bit.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "marching_steps_kats.json")))


@pytest.fixture(scope="module")
def shim():
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "kat_shim")], check=True)
    lib = C.CDLL(os.path.join(HERE, "kat_shim", "_build", "libdgmr_kat.so"))
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    lib.kat_density_array_f32.argtypes = [C.c_int, C.c_float, f32p, C.c_int, f32p, f32p]
    lib.kat_density_array_f64.argtypes = [C.c_int, C.c_double, f64p, C.c_int, f64p, f64p]
    lib.kat_density_combine_f32.argtypes = [f32p, f32p, f32p]
    lib.kat_density_combine_f64.argtypes = [f64p, f64p, f64p]
    lib.kat_density_sample16_f32.argtypes = [C.c_float, f32p, C.c_int, f32p]
    lib.kat_density_randomised_f32.argtypes = [C.c_int] * 3
    lib.kat_density_randomised_f64.argtypes = [C.c_int] * 3
    lib.kat_pl_sample.argtypes = [f64p, C.c_double, f64p]
    lib.kat_pl_valid.argtypes = [f64p]
    lib.kat_pl_create.argtypes = [f64p, f64p, f64p, f64p, C.c_double, f64p]
    lib.kat_pl_volume_integrate.argtypes = [f64p, C.c_int, C.c_int, f64p]
    lib.kat_rbs4.argtypes = [C.c_float, C.c_float, f32p, C.c_int, i32p, i32p, f32p, f32p]
    lib.kat_pl_create_oracle.argtypes = lib.kat_pl_create.argtypes
    lib.kat_pl_volume_integrate_oracle.argtypes = lib.kat_pl_volume_integrate.argtypes
    lib.kat_rbs4_oracle.argtypes = lib.kat_rbs4.argtypes
    lib.kat_compare_sizers.argtypes = [C.c_uint, C.c_int]
    lib.kat_compare_sizers.restype = C.c_long
    lib.kat_compare_fits.argtypes = [C.c_uint, C.c_int]
    lib.kat_compare_fits.restype = C.c_long
    lib.kat_compare_warp_sizer.argtypes = [C.c_uint, C.c_int]
    lib.kat_compare_warp_sizer.restype = C.c_long
    return lib


# the bin fit and bin sizer exist twice: the product's device header (csrc/dgmr_volume_fit.h)
# and the oracle's own restatement (oracle/dgmr_oracle_volume_fit.h); the KATs pin both
VF_IMPLS = ["product", "oracle"]


def vf(shim, name, impl):
    return getattr(shim, name if impl == "product" else name + "_oracle")


def value(lit: str, dtype):
    """A C++ numeric literal converted the way the test's scalar_t sees it."""
    if lit.endswith("f"):
        v = np.float32(lit[:-1])
        return dtype(v)
    return dtype(np.float64(lit))


# ---------------------------------------------------------------- DensityArray KATs
class Runner:
    def __init__(self, impl, dtype, shim=None):
        self.impl, self.dtype, self.shim = impl, dtype, shim

    def puts(self, cap, start, entries):
        dt = self.dtype
        if self.impl == "oracle":
            secs, end = O.density_array(cap, dt(start), [list(e) for e in entries], dt)
            return secs, end
        ops = np.ascontiguousarray(np.asarray(entries, dtype=dt).reshape(-1)) if entries else np.zeros(3, dt)
        out = np.zeros(48, dt)
        end = np.zeros(1, dt)
        fn = self.shim.kat_density_array_f32 if dt == np.float32 else self.shim.kat_density_array_f64
        n = fn(cap, dt(start), ops, len(entries), out, end)
        return out[:3 * n].reshape(n, 3), float(end[0])

    def combine(self, a, b):
        dt = self.dtype
        if self.impl == "oracle":
            return O.density_combine(np.asarray(a, dt), np.asarray(b, dt), dt)
        out = np.zeros(9, dt)
        fn = self.shim.kat_density_combine_f32 if dt == np.float32 else self.shim.kat_density_combine_f64
        fn(np.asarray(a, dt), np.asarray(b, dt), out)
        return out.reshape(3, 3)


FIELDS = {"start": 0, "end": 1, "delta_t": 2}


@pytest.mark.parametrize("impl", ["oracle", "product"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("section", KATS["sections"], ids=[s["name"] for s in KATS["sections"]])
def test_density_array_kats(section, dtype, impl, shim):
    r = Runner(impl, dtype, shim)
    cap = start = None
    entries = []
    v = None
    n_checks = 0
    for op in section["ops"]:
        kind = op["op"]
        if kind == "combine":
            v = r.combine([value(x, dtype) for x in op["a"]], [value(x, dtype) for x in op["b"]])
        elif kind == "vfield":
            assert v[op["index"], FIELDS[op["field"]]] == value(op["value"], dtype), op
            n_checks += 1
        elif kind == "array":
            cap, start, entries = op["capacity"], value(op["start"], dtype), []
        elif kind == "put":
            entries.append([value(x, dtype) for x in op["entry"]])
        elif kind in ("size", "field"):
            secs, _ = r.puts(cap, start, entries)
            if kind == "size":
                assert len(secs) == op["value"], (op, secs)
            else:
                assert secs[op["index"], FIELDS[op["field"]]] == value(op["value"], dtype), (op, secs)
            n_checks += 1
    assert n_checks > 0


def test_kat_fixture_is_complete():
    n = sum(1 for s in KATS["sections"] for o in s["ops"] if o["op"] in ("size", "field", "vfield"))
    assert len(KATS["sections"]) == 20 and n == 484


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_density_array_randomised_oracle(dtype):
    assert O.density_randomised(1000, 100, 50, dtype) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_density_array_randomised_product(dtype, shim):
    fn = shim.kat_density_randomised_f32 if dtype == np.float32 else shim.kat_density_randomised_f64
    assert fn(1000, 100, 50) == 0


# unittests/marching_steps.cpp:28-66
def test_sampler_empty_and_filled(shim):
    for impl in ("oracle", "product"):
        empty = (O.density_sample(4, np.float32(0.1), [], 16) if impl == "oracle" else None)
        if impl == "product":
            empty = np.zeros(16, np.float32)
            shim.kat_density_sample16_f32(np.float32(0.1), np.zeros(3, np.float32), 0, empty)
        assert np.all(empty == 0)
        puts = [[0.2, 1.0, 0.1], [1.0, 2.0, 0.2], [2.0, 2.5, 0.5], [3.0, 4.0, 1.0]]
        p32 = [[np.float32(x) for x in e] for e in puts]
        if impl == "oracle":
            smp = O.density_sample(4, np.float32(0.1), p32, 16)
        else:
            smp = np.zeros(16, np.float32)
            shim.kat_density_sample16_f32(np.float32(0.1), np.asarray(p32, np.float32).reshape(-1), 4, smp)
        secs, _ = O.density_array(4, np.float32(0.1), p32)
        assert smp[0] == np.float32(0.2)

        def target(t):
            for s in secs:
                if s[0] <= t < s[1]:
                    return s[2]
            return np.inf

        for i in range(1, 16):
            d = smp[i] - smp[i - 1]
            assert d > 0
            t = smp[i - 1]
            while t < smp[i]:
                assert d <= target(t) + 0.001
                t = np.float32(t + np.float32(0.01))


# ---------------------------------------------------------------- piecewise linear
def pack(d0, k0, t1, t2, k2, t_right=0.0):
    return np.asarray(list(d0) + list(k0) + list(t1) + list(t2) + list(k2) + [t_right], np.float64)


def test_piecewise_linear_function_group(shim):
    f = pack((0.8, 0.4, 0.5, 0.2), (-0.8, -0.2, 0.5, 0.0), (1.0, 2.0, 0.5, 2.0), (2.0, 2.0, 0.5, 2.0), (0.1, 0.2, 0.3, 0.4))
    assert shim.kat_pl_valid(f) == 1
    expect = {0.0: (0.8, 0.4, 0.50, 0.2), 0.5: (0.4, 0.3, 0.75, 0.2), 1.0: (0.0, 0.2, 0.90, 0.2),
              2.0: (0.0, 0.0, 1.20, 0.2), 3.0: (0.1, 0.2, 1.50, 0.6)}
    out = np.zeros(4)
    for t, e in expect.items():
        shim.kat_pl_sample(f, t, out)
        assert np.array_equal((out * 1000.0).astype(np.int32), (np.asarray(e) * 1000.0).astype(np.int32)), (t, out)


@pytest.mark.parametrize("case", [
    dict(mpl=(0.8, 0.4, 0.5, 0.2), mt=(0.3, 0.6, 0.3, 0.8), el=(0.4, 0.7, 0.2, 0.9), er=(0.2, 0.1, 0.0, 0.1), tr=0.8, td=0.001,
         rounding=0.0),
    dict(mpl=(0.5, 0.5, 0.5, 0.5), mt=(0.8, 0.8, 0.8, 0.0), el=(0.0, 0.0, 0.2, 0.0), er=(0.0, 0.1, 0.0, 0.0), tr=0.8, td=0.000001,
         rounding=0.5),
])
@pytest.mark.parametrize("impl", VF_IMPLS)
def test_piecewise_linear_fit_conserves_mass(shim, case, impl):
    f = np.zeros(21)
    a = lambda v: np.asarray(v, np.float64)
    vf(shim, "kat_pl_create", impl)(a(case["mpl"]), a(case["mt"]), a(case["el"]), a(case["er"]), case["tr"], f)
    assert shim.kat_pl_valid(f) == 1
    out = np.zeros(4)
    shim.kat_pl_sample(f, 0.0, out)
    assert np.array_equal((out * 1000 + 0.5).astype(np.int32), (a(case["el"]) * 1000 + 0.5).astype(np.int32))
    shim.kat_pl_sample(f, case["tr"], out)
    assert np.array_equal((out * 1000 + 0.5).astype(np.int32), (a(case["er"]) * 1000 + 0.5).astype(np.int32))
    # numeric mass: vectorised sample of the piecewise model over [0, t_right)
    td = case["td"]
    t = np.arange(0.0, case["tr"], td)
    d0, k0, t1, t2, k2 = f[0:4], f[4:8], f[8:12], f[12:16], f[16:20]
    T = t[:, None]
    vals = np.where(T <= t1, d0 + k0 * T, np.where(T <= t2, 0.0, d0 + t1 * k0 + (T - t2) * k2))
    mass = vals.sum(axis=0) * td
    assert np.array_equal((mass * 1000 + case["rounding"]).astype(np.int32),
                          (a(case["mt"]) * 1000 + case["rounding"]).astype(np.int32)), mass


@pytest.mark.parametrize("impl", VF_IMPLS)
def test_piecewise_linear_volume_integral(shim, impl):
    rows = [
        ((0.0, 0.0, 0.0, 0.0), (0.3, 0.6, 0.3, 0.6), (0.0, 0.0, 0.0, 0.0), (0.2, 0.1, 0.0, 0.1), 0.8),
        ((0.8, 0.4, 0.5, 0.3), (0.5, 0.4, 0.8, 0.2), (0.2, 0.1, 0.0, 0.1), (0.4, 0.7, 0.2, 0.9), 0.5),
        ((0.6, 0.7, 0.1, 0.8), (0.1, 0.0, 0.1, 0.1), (0.4, 0.7, 0.2, 0.9), (0.8, 0.1, 0.8, 0.7), 1.5),
        ((0.1, 0.8, 0.7, 0.5), (0.1, 0.2, 0.0, 0.2), (0.8, 0.1, 0.8, 0.7), (0.4, 0.7, 0.2, 0.1), 2.5),
        ((0.5, 0.2, 0.6, 0.3), (0.5, 0.6, 0.7, 0.7), (0.4, 0.7, 0.2, 0.1), (0.4, 0.7, 0.2, 0.2), 0.5),
        ((0.7, 0.8, 0.2, 0.5), (0.5, 0.2, 0.3, 0.5), (0.4, 0.7, 0.2, 0.2), (0.4, 0.7, 0.2, 1.9), 0.8),
        ((0.8, 0.4, 0.8, 0.2), (0.3, 1.6, 1.3, 1.9), (0.4, 0.7, 0.2, 1.9), (0.4, 0.7, 0.2, 0.5), 0.1),
        ((0.1, 0.1, 0.4, 0.9), (0.8, 0.7, 0.3, 2.4), (0.4, 0.7, 0.2, 0.5), (0.2, 0.1, 0.0, 0.1), 1.2),
    ]
    a = lambda v: np.asarray(v, np.float64)
    groups = []
    for mpl, mt, el, er, tr in rows:
        f = np.zeros(21)
        vf(shim, "kat_pl_create", impl)(a(mpl), a(mt), a(el), a(er), tr, f)
        groups.append(f)
    packed = np.ascontiguousarray(np.concatenate(groups))
    out = np.zeros(3)
    vf(shim, "kat_pl_volume_integrate", impl)(packed, 8, 256, out)
    # numeric reference (Eq. 15 of the reference test): 1e6 steps over all bins
    n_ref = 1_000_000
    max_t = sum(r[4] for r in rows)
    dt = max_t / n_ref
    t = np.arange(n_ref) * dt
    bounds = np.cumsum([0.0] + [r[4] for r in rows])
    vals = np.zeros((n_ref, 4))
    for i, f in enumerate(groups):
        m = (t >= bounds[i]) & (t < bounds[i + 1]) if i < 7 else (t >= bounds[i])
        tt = (t[m] - bounds[i])[:, None]
        d0, k0, t1, t2, k2 = f[0:4], f[4:8], f[8:12], f[12:16], f[16:20]
        vals[m] = np.where(tt <= t1, d0 + k0 * tt, np.where(tt <= t2, 0.0, d0 + t1 * k0 + (tt - t2) * k2))
    cum_m = np.concatenate([[0.0], np.cumsum(vals[:, 3] * dt)[:-1]])
    ref = (vals[:, :3] * np.exp(-cum_m)[:, None] * dt).sum(axis=0)
    assert 0.0 < cum_m[-1] + vals[-1, 3] * dt < 20.0
    assert np.all(ref >= 0) and np.all(ref < 2.0)
    assert np.all(np.abs(out - ref) < 1.0 / 256), (out, ref)


# ---------------------------------------------------------------- RasterBinSizer
RBS_CASES = {
    "start empty": [],
    "single opaque gaussian": [(10.52, 8, 4)],
    "bad gaussian order": [(0.25, 10, 2), (0.25, 8, 1), (0.25, 6, 2), (0.25, 4, 1), (0.25, 2, 2), (0.25, 0, 1)],
    "only one gaussian at 0.6 opacity": [(0.6, 10, 2)],
    "only one gaussian at 0.3 opacity": [(0.3, 10, 2)],
    "several gaussians, filling up": [(0.35, 1.3, 1.0), (0.40, 4.7, 0.81), (0.6, 6.8, 1.0), (10.8, 9.6, 0.25)],
    "one gap in transmission stops": [(0.7, 4.7, 0.81), (0.6, 6.8, 1.0), (0.8, 9.6, 0.25)],
    "one gap in transmission stops, random order": [(0.7, 4.7, 0.81), (0.8, 9.6, 0.25), (0.6, 6.8, 1.0)],
    "two gaps in transmission stops": [(0.6, 6.8, 1.0), (0.9, 9.6, 0.25)],
    "many small, random order": [(0.08, 1.8, 1.33), (0.05, 4.6, 0.25), (0.18, 2.8, 1.22), (0.06, 5.0, 0.33), (0.08, 3.8, 1.45),
                                 (0.23, 9.6, 0.25), (0.18, 6.0, 1.20), (0.05, 4.6, 0.25), (0.21, 6.8, 1.00), (0.38, 10.2, 0.25),
                                 (0.26, 10.8, 1.00), (0.28, 10.3, 0.25), (0.21, 10.5, 1.00), (0.37, 10.9, 0.25)],
}
# is_full() expectations stated by the reference sections (after each add, after finalise)
RBS_FULL = {
    "start empty": ([], False),
    "single opaque gaussian": ([True], True),
    "bad gaussian order": ([False] * 6, False),
    "only one gaussian at 0.6 opacity": ([False], False),
    "several gaussians, filling up": ([False, False, False, True], None),
}


@pytest.mark.parametrize("impl", VF_IMPLS)
@pytest.mark.parametrize("name", list(RBS_CASES))
def test_raster_bin_sizer(shim, name, impl):
    adds = np.asarray(RBS_CASES[name], np.float32).reshape(-1)
    n = len(RBS_CASES[name])
    full = np.zeros(max(n, 1), np.int32)
    full_fin = np.zeros(1, np.int32)
    b = np.zeros(4, np.float32)
    e = np.zeros(4, np.float32)
    # test configuration of unittests/raster_bin_sizer.cpp:29-33: 4 bins, threshold 0.1, relevance 1 sigma
    vf(shim, "kat_rbs4", impl)(np.float32(1.0), np.float32(0.1), adds if n else np.zeros(3, np.float32), n, full, full_fin,
                               b, e)
    assert b[0] == pytest.approx(0.0)
    for i in range(3):
        assert e[i] == pytest.approx(b[i + 1])
    for i in range(4):
        assert b[i] <= e[i]
    if name == "start empty":
        assert np.allclose(b, 0) and np.allclose(e, 0)
    if name in RBS_FULL:
        exp_adds, exp_fin = RBS_FULL[name]
        assert [bool(x) for x in full[:n]] == exp_adds
        if exp_fin is not None:
            assert bool(full_fin[0]) == exp_fin


def test_oracle_and_product_bin_sizers_agree(shim):
    """20k random add sequences (32 and 4 bins): saturation after every add
    and the final borders, bit for bit."""
    assert shim.kat_compare_sizers(7, 10000) == 0


def test_warp_parallel_bin_sizer_matches_the_one_thread_sizer(shim):
    """The volume rasteriser's warp form of the sizer (one slot per lane: the
    insertion position from a ballot, merge costs priced lane-parallel, the
    first of equal minimum costs), emulated lane by lane: 20k random add
    sequences give the one-thread RasterBinSizer's saturation flags and final
    borders bit for bit."""
    assert shim.kat_compare_warp_sizer(5, 20000) == 0


def test_oracle_and_product_bin_fits_agree(shim):
    """200k random four-channel bin fits: all five parameters of every
    channel, bit for bit."""
    assert shim.kat_compare_fits(11, 200000) == 0


# ---------------------------------------------------------------- math.h helpers
@pytest.mark.parametrize("which,inputs", [
    # unittests/math.cpp:96-106: every permutation of (1, 2, 3) -> {2, 3}
    ("larger", [(1, 2, 3), (1, 3, 2), (2, 3, 1), (2, 1, 3), (3, 2, 1), (3, 1, 2)]),
    # unittests/math.cpp:107-117: every permutation of (2, 3, 4) -> {2, 3}
    ("smaller", [(4, 2, 3), (4, 3, 2), (2, 3, 4), (2, 4, 3), (3, 2, 4), (3, 4, 2)]),
])
def test_larger2_smaller2_kats(which, inputs):
    """The oracle's larger2 / smaller2 (math.h:112-155) on the reference's
    known answers: the pair is (2, 3) in either order."""
    out = O.pick2(which, inputs)
    for row in out:
        assert sorted(row.tolist()) == [2.0, 3.0]


def test_larger2_smaller2_pick_the_extremes():
    """On random scale triples (ties included) larger2 drops a smallest
    component and smaller2 a largest one, as the Ots / Ols formulations use
    them (math.h:284-293)."""
    rng = np.random.default_rng(5)
    v = rng.integers(1, 5, size=(4000, 3)).astype(np.float32)
    lg, sm = O.pick2("larger", v), O.pick2("smaller", v)
    srt = np.sort(v, axis=1)
    assert np.array_equal(np.sort(lg, axis=1), srt[:, 1:])
    assert np.array_equal(np.sort(sm, axis=1), srt[:, :2])


# ---------------------------------------------------------------- elementary functions
def test_deterministic_exp_log_erf_error_bounds():
    import math
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-100, 80, 20000), rng.uniform(-2, 2, 20000), [0.0, -1e-8, 1e-8, 88.0, -87.0]]).astype(np.float32)
    ref = np.array([math.exp(float(v)) for v in x])
    got = O.fmath("exp", x).astype(np.float64)
    ok = ref > 1.2e-38
    assert np.max(np.abs(got[ok] - ref[ok]) / ref[ok]) < 4e-7
    xl = np.concatenate([rng.uniform(1e-30, 1e30, 10000), rng.uniform(0.5, 2.0, 10000), rng.uniform(1e-6, 1.0, 10000)]).astype(np.float32)
    refl = np.array([math.log(float(v)) for v in xl])
    gotl = O.fmath("log", xl).astype(np.float64)
    assert np.max(np.abs(gotl - refl) / np.maximum(np.abs(refl), 1e-3)) < 4e-7
    xe = rng.uniform(-6, 6, 20000).astype(np.float32)
    refe = np.array([math.erf(float(v)) for v in xe])
    gote = O.fmath("erf", xe).astype(np.float64)
    assert np.max(np.abs(gote - refe)) < 2.5e-7  # Abramowitz & Stegun 7.1.26 bound 1.5e-7 plus float rounding


# windows swept ulp by ulp: the 1/255 cutoffs (exp near ln(1/255), log near
# 255), the branch points of each routine (log's sqrt(2) split and 1, erf's
# series / Hastings switch at 1 and its saturation at 3.92) and the ends of
# exp's range (its reduction's rounding switch at +-ln2/2, gradual underflow,
# the 2^127 split, overflow).  Every float input was also compared once, all
# 2^32 of them, with no difference.
FMATH_WINDOWS = {
    "exp": [(-5.6, -5.5), (-0.36, -0.33), (0.33, 0.36), (-88.0, -86.9), (-104.1, -103.9), (88.3, 88.75)],
    "log": [(0.99, 1.01), (1.41, 1.42), (0.70, 0.71), (254.0, 256.0), (1e-39, 2e-38)],
    "erf": [(-1.01, -0.99), (0.99, 1.01), (3.91, 3.93), (-3.93, -3.91)],
}


@pytest.mark.parametrize("which", ["exp", "log", "erf"])
def test_oracle_and_product_elementary_functions_agree(shim, which):
    """The oracle compiles no product source: its exp / log / erf are its own
    coding (oracle/dgmr_oracle_fmath.h) of the methods csrc/dgmr_fmath.h
    follows.  Every 257th float bit pattern (both signs, every exponent, NaN,
    infinities; ~16.7M inputs) and every float of the windows above must give
    the same bits from both (NaN payloads aside)."""
    f = shim.kat_fmath_mismatches
    f.restype = C.c_long
    f.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_float, C.c_float, C.POINTER(C.c_long)]
    w = {"exp": 0, "log": 1, "erf": 2}[which]
    n = C.c_long(0)
    assert f(w, 0, 257, 1.0, 0.0, C.byref(n)) == 0
    total = n.value
    for lo, hi in FMATH_WINDOWS[which]:
        assert f(w, 0, 0xFFFFFFFF, lo, hi, C.byref(n)) == 0, (lo, hi)
        total += n.value
    assert total > 16_000_000


def test_erf_reciprocal_is_the_correctly_rounded_division(shim):
    """erf_f's 7.1.26 branch takes 1 / (1 + 0.3275911 |x|) for 1 <= |x| < 3.92
    from fused multiply-adds (recip_hastings): for every float in a range that
    holds all those divisors it must equal 1.0f / d bit for bit, so erf_f gives
    the same bits as with the division (and as the oracle, which divides)."""
    f = shim.kat_recip_mismatches
    f.restype = C.c_long
    f.argtypes = [C.c_float, C.c_float, C.POINTER(C.c_long)]
    n = C.c_long(0)
    assert f(1.326, 2.286, C.byref(n)) == 0
    assert n.value > 6_000_000


@pytest.mark.parametrize("suffix", ["f32", "f64"])
def test_insertions_claimed_unchanged_leave_the_set_unchanged(shim, suffix):
    """The volume marcher skips a section insertion that
    SectionSet::put_leaves_unchanged accepts (its device form tests the same
    conditions lane-parallel).  On random insertion sequences built to make
    equal ends and equal steps common, every accepted insertion must leave the
    set bit for bit as it was, and a good share of insertions must be accepted."""
    f = getattr(shim, f"kat_section_unchanged_{suffix}")
    f.restype = C.c_long
    f.argtypes = [C.c_uint, C.c_int, C.POINTER(C.c_long)]
    covered = C.c_long(0)
    bad = f(11, 20000, C.byref(covered))
    assert bad == 0
    assert covered.value > 100000


@pytest.mark.parametrize("suffix", ["f32", "f64"])
def test_insertion_by_pieces_equals_put(shim, suffix):
    """The marcher's warps insert a section as SectionSet::merge_pieces plus a
    lane-parallel move of the kept tail (put_by_pieces is its serial form)
    instead of put()'s ring walk.  On random insertion sequences (capacities 16
    and 4, so full sets and cuts are common) both must leave the same set, bit
    for bit, after every insertion."""
    f = getattr(shim, f"kat_section_by_pieces_{suffix}")
    f.restype = C.c_long
    f.argtypes = [C.c_uint, C.c_int, C.POINTER(C.c_long)]
    merges = C.c_long(0)
    assert f(5, 20000, C.byref(merges)) == 0
    assert merges.value > 1000000


@pytest.mark.parametrize("suffix", ["f32", "f64"])
def test_sample_positions_by_sections_equal_the_serial_walk(shim, suffix):
    """The marcher's warps place a large step's 128 samples section by section
    (each section's chain on its own lane, after the samples of the sections
    before it; sample_positions_by_sections is the serial form).  On random
    section sets, some with steps so small that the 128-sample cap cuts a
    section short, the positions must be sample_positions_n's, bit for bit."""
    f = getattr(shim, f"kat_samples_by_sections_{suffix}")
    f.restype = C.c_long
    f.argtypes = [C.c_uint, C.c_int, C.POINTER(C.c_long)]
    sets = C.c_long(0)
    assert f(13, 30000, C.byref(sets)) == 0
    assert sets.value > 100000


def test_range_specialised_exp_is_bit_identical(shim):
    """The blend's exp_f_nonpos must return exp_f's bits for every input."""
    f = shim.kat_exp_nonpos_mismatches
    f.restype = C.c_long
    f.argtypes = [C.c_float, C.c_float, C.c_uint]
    assert f(-100.0, 2.0, 97) == 0


def test_insertions_never_overflow_the_set(shim):
    """A section set holds at most 16 sections whatever is inserted: no
    insertion leaves more, or writes past the set (the marcher keeps one set
    per warp in shared memory, next to the other warps' data)."""
    f = shim.kat_section_overflows
    f.restype = C.c_long
    f.argtypes = [C.c_uint, C.c_int]
    assert f(3, 40000) == 0
