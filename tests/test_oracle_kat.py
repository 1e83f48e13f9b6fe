"""Known-answer and property tests of the CPU oracle, re-expressing the
reference's own GTest assertions (LucidRenderer/cpp_renderer/test/*) on the
restated functions.  These pin the oracle's component math to the
reference's tests; pixel-level parity has no reference fixture (the
reference pins no image or RNG values)."""
import ctypes
import math

import numpy as np
import pytest

EPS = 1e-4   # test_bsdf.cpp:21 kEps


def f3(*v):
    return np.array(v, dtype=np.float32)


# ---- test_bsdf.cpp:33-180 (Fresnel) -------------------------------------
def test_fresnel_schlick(oracle_lib):
    L = oracle_lib
    assert abs(L.orc_fresnel_schlick(0.0, 0.04) - 1.0) < EPS          # CosTheta0_ReturnsOne
    assert abs(L.orc_fresnel_schlick(1.0, 0.04) - 0.04) < EPS         # CosTheta1_ReturnsF0
    assert abs(L.orc_fresnel_schlick(1.0, 0.0)) < EPS                 # F0Zero
    assert abs(L.orc_fresnel_schlick(0.0, 0.0) - 1.0) < EPS
    for c in (1.0, 0.5, 0.0):
        assert abs(L.orc_fresnel_schlick(c, 1.0) - 1.0) < EPS         # F0One_AlwaysOne
    prev = L.orc_fresnel_schlick(0.0, 0.04)
    for c in np.arange(0.1, 1.0001, 0.1):                              # MonotonicDecrease
        cur = L.orc_fresnel_schlick(float(c), 0.04)
        assert cur <= prev + EPS
        prev = cur
    exp = 0.04 + (1 - 0.04) * 0.5 ** 5                                 # HalfAngle_ExpectedValue
    assert abs(L.orc_fresnel_schlick(0.5, 0.04) - exp) < EPS


def test_fresnel_dielectric(oracle_lib):
    L = oracle_lib
    exp = ((1.5 - 1.0) / (1.5 + 1.0)) ** 2
    assert abs(L.orc_fresnel_dielectric(1.0, 1.5) - exp) < EPS         # NormalIncidence
    assert abs(L.orc_fresnel_dielectric(1.0, 1.0 / 1.5) - exp) < EPS
    assert abs(L.orc_fresnel_dielectric(0.0, 1.5) - 1.0) < EPS         # GrazingAngle_One
    assert abs(L.orc_fresnel_dielectric(1.0, 1.0)) < EPS               # EtaOne_ZeroReflectance
    cos_i = math.sqrt(1 - 0.8 * 0.8)
    assert abs(L.orc_fresnel_dielectric(cos_i, 1.5) - 1.0) < EPS       # TotalInternalReflection
    r = L.orc_fresnel_dielectric(1.0, 1.5)
    assert 0.0 < r < 1.0                                              # BelowCriticalAngle


# ---- test_bsdf.cpp:193-306 (GGX) ----------------------------------------
def test_ggx(oracle_lib):
    L = oracle_lib
    assert L.orc_ggx_d(1.0, 0.5) > L.orc_ggx_d(0.9, 0.5)               # D_PeakAtNdotH1
    assert L.orc_ggx_d(1.0, 0.1) > L.orc_ggx_d(1.0, 0.5)               # smoother -> sharper peak
    for r in (0.01, 0.5, 1.0):
        g1 = L.orc_ggx_g1(1.0, r)
        assert 0.0 < g1 <= 1.0 + EPS                                   # G1 in (0, 1]
        assert L.orc_ggx_g2(0.0, 0.5, r) == 0.0                        # back-facing -> 0
        assert L.orc_ggx_g2(0.7, 0.6, r) <= min(L.orc_ggx_g1(0.7, r), L.orc_ggx_g1(0.6, r)) + EPS


# ---- test_integrator.cpp:36-130 (MIS, pdf helpers) ----------------------
def test_mis_power_heuristic(oracle_lib):
    L = oracle_lib
    lo, med, hi = 0.1, 0.5, 2.0
    assert L.orc_mis_power(hi, lo) > 0.9 and L.orc_mis_power(lo, hi) < 0.1
    for a, b in ((med, hi), (lo, hi), (lo, med)):
        assert abs(L.orc_mis_power(a, b) + L.orc_mis_power(b, a) - 1.0) < EPS
    assert abs(L.orc_mis_power(med, med) - 0.5) < EPS
    for a in (0.01, 0.1, 0.5, 1.0, 2.0, 10.0):
        for b in (0.01, 0.1, 0.5, 1.0, 2.0, 10.0):
            assert 0.0 <= L.orc_mis_power(a, b) <= 1.0
    assert abs(L.orc_mis_power(med, hi) - med * med / (med * med + hi * hi)) < EPS
    assert math.isfinite(L.orc_mis_power(med, 0.0)) and abs(L.orc_mis_power(med, 0.0) - 1.0) < 0.01
    assert math.isfinite(L.orc_mis_power(0.0, med))


def test_light_pdf_and_inverse_square(oracle_lib):
    L = oracle_lib
    assert abs(L.orc_pdfw_from_area(3.0, 4.0, 1.0) - 2.25) < EPS       # test_light.cpp:341-355
    assert L.orc_pdfw_from_area(3.0, 4.0, 0.0) == 0.0                  # grazing -> 0
    assert L.orc_pdfw_from_area(3.0, 0.0, 1.0) == 0.0                  # zero area -> 0
    assert abs(L.orc_inv_sq(2.0) - 0.25) < EPS
    assert L.orc_inv_sq(0.0) == 0.0


# ---- test_geometry.cpp (triangle / AABB / sphere) -----------------------
TRI = f3(0, 0, 0, 1, 0, 0, 0, 1, 0)


def isect(L, o, d, tmin=1e-4, tmax=1e30):
    uvt = np.zeros(3, np.float32)
    oa, da = f3(*o), f3(*d)   # keep the arrays alive across the call
    hit = L.orc_isect_tri(oa.ctypes.data, da.ctypes.data, TRI.ctypes.data, tmin, tmax, uvt.ctypes.data)
    return hit, uvt


def test_triangle_intersection(oracle_lib):
    L = oracle_lib
    h, uvt = isect(L, (0.25, 0.25, 1), (0, 0, -1))
    assert h and abs(uvt[2] - 1) < 1e-5 and abs(uvt[0] - 0.25) < 1e-5 and abs(uvt[1] - 0.25) < 1e-5
    h, uvt = isect(L, (0, 0, 1), (0, 0, -1))
    assert h and abs(uvt[0]) < 1e-5 and abs(uvt[1]) < 1e-5              # HitVertex0
    h, uvt = isect(L, (1, 0, 1), (0, 0, -1))
    assert h and abs(uvt[0] - 1) < 1e-5                                # HitVertex1
    h, uvt = isect(L, (0, 1, 1), (0, 0, -1))
    assert h and abs(uvt[1] - 1) < 1e-5                                # HitVertex2
    h, uvt = isect(L, (0.5, 0, 1), (0, 0, -1))
    assert h and abs(uvt[0] - 0.5) < 1e-5                              # HitEdge01
    assert not isect(L, (2, 2, 1), (0, 0, -1))[0]                      # MissOutside
    assert not isect(L, (0.25, 0.25, 1), (1, 0, 0))[0]                 # MissParallel
    assert not isect(L, (0.25, 0.25, 1), (0, 0, 1))[0]                 # MissBehind
    h, uvt = isect(L, (0.25, 0.25, -1), (0, 0, 1))
    assert h and abs(uvt[2] - 1) < 1e-5                                # HitFromBehind
    assert not isect(L, (0.25, 0.25, 1), (0, 0, -1), tmin=2.0)[0]      # TMinConstraint
    assert not isect(L, (0.25, 0.25, 1), (0, 0, -1), tmax=0.5)[0]      # TMaxConstraint


def test_aabb_intersection(oracle_lib):
    L = oracle_lib
    bmin, bmax = f3(-1, -1, -1), f3(1, 1, 1)

    def box(o, d):
        d = np.array(d, np.float64)
        d = (d / np.linalg.norm(d)).astype(np.float32)
        oa = f3(*o)
        return L.orc_isect_aabb(oa.ctypes.data, d.ctypes.data, bmin.ctypes.data, bmax.ctypes.data)
    assert box((0, 0, 5), (0, 0, -1))                                  # HitFromFront
    assert box((5, 0, 0), (-1, 0, 0))                                  # HitFromSide
    assert box((5, 5, 5), (-1, -1, -1))                                # HitDiagonal
    assert not box((0, 5, 5), (0, 0, -1))                              # MissAbove
    assert not box((5, 0, 5), (0, 0, -1))                              # MissSide
    assert box((0, 0, 0), (0, 0, 1))                                   # RayInsideBox
    assert box((-5, 0, 0), (1, 0, 0))                                  # ParallelToXAxis
    assert not box((-5, 2, 0), (1, 0, 0))                              # ParallelToXAxisMiss


def test_sphere_intersection(oracle_lib):
    L = oracle_lib
    c = f3(0, 0, 0)
    t = ctypes.c_float()

    def sph(o, d):
        oa, da = f3(*o), f3(*d)
        return L.orc_isect_sphere(oa.ctypes.data, da.ctypes.data, c.ctypes.data, 1.0, ctypes.byref(t))
    assert sph((0, 0, 5), (0, 0, -1)) and abs(t.value - 4.0) < 1e-5      # HitCenter
    assert not sph((0, 5, 5), (0, 0, -1))                               # MissFarAway
    assert sph((0, 0, 0), (0, 0, 1)) and abs(t.value - 1.0) < 1e-5       # RayInsideSphere
    assert not sph((0, 0, 5), (0, 0, 1))                                # RayBehindSphere


# ---- test_volume_phase.cpp (HG normalisation) ---------------------------
@pytest.mark.parametrize("g", [0.0, 0.3, -0.5, 0.8])
def test_hg_normalised(oracle_lib, g):
    L = oracle_lib
    rng = np.random.default_rng(1)
    n = 200000
    z = rng.uniform(-1, 1, n)                       # uniform on the sphere: pdf 1/(4 pi)
    vals = np.array([L.orc_hg_eval(g, float(c)) for c in z[:20000]])
    est = vals.mean() * 4 * math.pi
    assert abs(est - 1.0) < 0.03
    # sampled cosines follow the HG pdf (mean cosine = g)
    wo = f3(0, 0, 1)
    wi = np.zeros(3, np.float32)
    pdf = ctypes.c_float()
    u = rng.random((20000, 2))
    cs = []
    for a, b in u:
        L.orc_hg_sample(g, wo.ctypes.data, float(a), float(b), wi.ctypes.data, ctypes.byref(pdf))
        cs.append(float(wi[2]))
    assert abs(np.mean(cs) - g) < 0.02


# ---- test_random.cpp (statistics of the seeded PCG32 stream) ------------
def test_rng_statistics(oracle_lib):
    L = oracle_lib
    n = 4096
    u = np.zeros(n, np.uint32)
    f = np.zeros(n, np.float32)
    allf = []
    for s in range(8):
        L.orc_rng_sequence(3, 7, s, n, u.ctypes.data, f.ctypes.data)
        assert np.all(f >= 0.0) and np.all(f < 1.0)
        assert np.array_equal(f, (u >> 9).astype(np.float32) * np.float32(2.0 ** -23))
        allf.append(f.copy())
    allf = np.concatenate(allf)
    assert abs(allf.mean() - 0.5) < 0.01
    assert abs(allf.var() - 1 / 12) < 0.005
    hist = np.histogram(allf, bins=16, range=(0, 1))[0]
    assert hist.min() > 0.8 * len(allf) / 16
    # different pixels / samples decorrelate
    a = np.zeros(n, np.uint32); b = np.zeros(n, np.uint32)
    L.orc_rng_sequence(0, 0, 0, n, a.ctypes.data, f.ctypes.data)
    L.orc_rng_sequence(1, 0, 0, n, b.ctypes.data, f.ctypes.data)
    assert np.mean(a == b) < 0.01


def test_deterministic_math_accuracy(oracle_lib):
    """lucid_math.h (shared by oracle and kernels) vs float64 libm."""
    L = oracle_lib
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(0, 2 * math.pi, 20000), np.float32(2 * math.pi) * rng.random(200)])
    for fn, ref in ((0, np.sin), (1, np.cos)):
        got = np.array([L.orc_lm(fn, float(x)) for x in xs], np.float32)
        want = ref(xs.astype(np.float32).astype(np.float64))
        err = np.abs(got.astype(np.float64) - want)
        assert err.max() < 2.5e-7, (fn, err.max())
    e = rng.uniform(-80, 0, 20000).astype(np.float32)
    got = np.array([L.orc_lm(2, float(x)) for x in e], np.float32).astype(np.float64)
    want = np.exp(e.astype(np.float64))
    assert np.max(np.abs(got - want) / want) < 2.4e-7
    lg = rng.uniform(1e-12, 1.0, 20000).astype(np.float32)
    got = np.array([L.orc_lm(3, float(x)) for x in lg], np.float32).astype(np.float64)
    want = np.log(lg.astype(np.float64))
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-30)) < 2.4e-7
