"""Pins of the FP64 CPU oracle (oracle/rf_oracle.c).

The reference ships no golden vectors for this path (parity unpinned against
reference output), so the oracle is pinned by: rnglib against the published
L'Ecuyer-Cote recurrences in exact integer arithmetic; closed-form known
answers (cm_COS single term, spectra_RF.f90:210-220); the contraction recast
against the direct sum; ensemble moments of the discrete spectral sum; and
the reference's formulas for the marginal map, normalisation and partition of
unity.  Small sizes: the whole file runs in seconds.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import grid, uniform_points

M1, M2 = 2147483563, 2147483399
PI = 3.1415926535898  # constants_RF.f90:5


def lecuyer(seed_start, count):
    """Independent restatement: i4_uni values of generator 1 seeded with
    (72 + 18 s, 72 + 18 s + 37), in exact integer arithmetic."""
    s1 = 72 + 18 * seed_start
    s2 = s1 + 37
    out = []
    for _ in range(count):
        s1 = 40014 * s1 % M1
        s2 = 40692 * s2 % M2
        z = s1 - s2
        if z < 1:
            z += M1 - 1
        out.append(z)
    return out


# ---------------------------------------------------------------- rnglib
def test_multmod_matches_exact_product():
    L = O.lib()
    rs = np.random.RandomState(0)
    for m in (M1, M2):
        for _ in range(2000):
            a = int(rs.randint(1, m))
            s = int(rs.randint(1, m))
            assert L.rfo_multmod(a, s, m) == a * s % m


def test_rnglib_constants_are_published_powers():
    # init_generator's a^(2^w) with w = 30 and set_initial_seed's a^(2^(v+w))
    # with v + w = 50 (rnglib.f90:840-841, :1559-1560)
    assert pow(40014, 2 ** 30, M1) == 1033780774 and pow(40692, 2 ** 30, M2) == 1494757890
    assert pow(40014, 2 ** 50, M1) == 2082007225 and pow(40692, 2 ** 50, M2) == 784306273


@pytest.mark.parametrize("seed_start", [0, 1, 7, 12345])
def test_i4_uni_stream(seed_start):
    L = O.lib()
    r = O.rng(seed_start)
    got = [L.rfo_rng_i4_uni(C.byref(r)) for _ in range(5000)]
    assert got == lecuyer(seed_start, 5000)


def test_r8_uni_01_scale():
    L = O.lib()
    r = O.rng(3)
    ref = lecuyer(3, 100)
    for z in ref:
        assert L.rfo_rng_r8_uni_01(C.byref(r)) == z * 4.656613057e-10


def test_initialize_default_seeds_and_generators():
    r = O.rng(None)
    assert (r.ig1[0], r.ig2[0]) == (1234567890, 123456789)
    ig1, ig2 = 1234567890, 123456789
    for g in range(1, 32):
        ig1 = 2082007225 * ig1 % M1
        ig2 = 784306273 * ig2 % M2
        assert (r.ig1[g], r.ig2[g]) == (ig1, ig2)
        assert (r.cg1[g], r.cg2[g]) == (ig1, ig2)


def test_advance_state_equals_repeated_draws():
    L = O.lib()
    a = O.rng(5)
    b = O.rng(5)
    L.rfo_rng_advance_state(C.byref(a), 6)
    for _ in range(64):
        L.rfo_rng_i4_uni(C.byref(b))
    assert (a.cg1[0], a.cg2[0]) == (b.cg1[0], b.cg2[0])


def test_init_generator_new_seed_jumps_2_pow_30():
    L = O.lib()
    r = O.rng(0)
    L.rfo_rng_init_generator(C.byref(r), 2)
    assert r.cg1[0] == pow(40014, 2 ** 30, M1) * 72 % M1
    assert r.cg2[0] == pow(40692, 2 ** 30, M2) * 109 % M2


# ------------------------------------------------------------ geometry
def test_shinozuka_geometry_reference_rule():
    x = grid(32, 0.1)
    g = O.OracleRequest(x, Nmc=1).geometry()
    # xRange = 3.1 -> kDelta = 2 pi / 3.41 = 1.8426 -> kNStep = 1 + ceil(7.355/1.8426) = 5
    assert list(g.kNStep) == [5, 5, 5]
    assert g.K == 125 * 4
    assert g.kDelta[0] == pytest.approx(7.355 / 4)
    assert g.ampMult == pytest.approx(2 * math.sqrt((7.355 / 4) ** 3 / (2 * PI) ** 3))
    g16 = O.OracleRequest(x, Nmc=1, kNStep=(16, 16, 16)).geometry()
    assert g16.K == 16 ** 3 * 4 and g16.kDelta[2] == pytest.approx(7.355 / 15)


def test_kpoints_quadrants_and_spectrum():
    x = grid(8, 0.2)
    rq = O.OracleRequest(x, Nmc=1, kNStep=(3, 4, 5))
    kp, amp, S = rq.kpoints()
    g = rq.geometry()
    assert kp.shape == (3 * 4 * 5 * 4, 3)
    base = 3 * 4 * 5
    signs = [(1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1)]  # set_kSign rows
    for q, sg in enumerate(signs):
        for b in range(base):
            i1, i2, i3 = b % 3, (b // 3) % 4, b // 12
            want = np.array([i1 * g.kDelta[0], i2 * g.kDelta[1], i3 * g.kDelta[2]]) * sg
            np.testing.assert_array_equal(kp[q * base + b], want)
    # per-axis product in axis order, as spectra_RF.f90:205-207 forms it
    want_S = np.ones(len(kp))
    for d in range(3):
        want_S = want_S * np.exp(-(kp[:, d] ** 2) / (4 * PI))
    np.testing.assert_allclose(S, want_S, rtol=1e-15)
    np.testing.assert_allclose(amp, np.sqrt(S), rtol=1e-15)


def test_literal_first_quadrant_unwritten():
    x = grid(8, 0.2)
    kp, _, S = O.OracleRequest(x, Nmc=1, kNStep=(3, 3, 3), literal=True).kpoints()
    assert np.all(kp[:27] == 0.0) and np.all(S[:27] == 1.0)
    assert np.any(kp[27:] != 0.0)


# ----------------------------------------------------------- known answers
def test_cm_cos_single_term_known_answer():
    """cm_COS: S = 1 at the 6th wavevector only, so the field is exactly
    ampMult * cos(k6 . x + phi6) (spectra_RF.f90:210-220)."""
    x = grid(6, 0.3)
    Nmc = 3
    rq = O.OracleRequest(x, corrMod=O.CM_COS, Nmc=Nmc, kNStep=(8, 3, 3))
    g = rq.geometry()
    f = rq.generate()
    z = lecuyer(0, g.K * Nmc)
    k6 = np.array([5 * g.kDelta[0], 0.0, 0.0])  # base grid index 5, first quadrant
    for r in range(Nmc):
        phi = 2.0 * PI * (z[r * g.K + 5] * 4.656613057e-10)
        want = g.ampMult * np.cos(x @ k6 + phi)
        np.testing.assert_allclose(f[r], want, rtol=0, atol=1e-14)


def test_cm_cos_literal_is_constant():
    """Literal mode: the 6th wavevector lies in the unwritten first quadrant,
    so the field is the constant ampMult * cos(phi6) (B2)."""
    x = grid(5, 0.3)
    rq = O.OracleRequest(x, corrMod=O.CM_COS, Nmc=2, kNStep=(8, 3, 3), literal=True)
    g = rq.geometry()
    f = rq.generate()
    z = lecuyer(0, g.K * 2)
    for r in range(2):
        phi = 2.0 * PI * (z[r * g.K + 5] * 4.656613057e-10)
        np.testing.assert_allclose(f[r], g.ampMult * np.cos(phi), rtol=0, atol=1e-14)


# ------------------------------------------------------- recast identity
@pytest.mark.parametrize("nDim,method", [(3, O.SHINOZUKA), (2, O.SHINOZUKA), (1, O.SHINOZUKA),
                                         (3, O.ISOTROPIC), (2, O.ISOTROPIC)])
def test_recast_equals_direct(nDim, method):
    x = uniform_points(300, 4.0, nDim=nDim, seed=nDim)
    kw = dict(kNStep=(6, 5, 4)) if method == O.SHINOZUKA else dict(isoNRadial=12, isoNDir=7)
    rq = O.OracleRequest(x, Nmc=3, method=method, corrL=(1.0, 0.7, 1.3), **kw)
    a = rq.generate()
    b = rq.generate(recast=True)
    np.testing.assert_allclose(b, a, rtol=0, atol=1e-12 * np.abs(a).max())


def test_rows_subset_matches_full():
    x = uniform_points(500, 3.0, seed=5)
    rq = O.OracleRequest(x, Nmc=2, kNStep=(5, 5, 5))
    full = rq.generate()
    rows = np.array([0, 7, 99, 499])
    np.testing.assert_array_equal(rq.generate(rows=rows), full[:, rows])


# ----------------------------------------------------------- statistics
def test_shinozuka_ensemble_variance_and_correlation():
    """Over realizations, Var f = ampMult^2/2 sum S_k and
    Cov(f(x), f(x+h e1)) = ampMult^2/2 sum S_k cos(k1 h) (random phases);
    the latter approaches exp(-pi h^2) (statistics_RF.f90:18-174, :425-443)."""
    h = 0.25
    pts = np.array([[0.0, 0.0, 0.0], [h, 0.0, 0.0], [2 * h, 0.0, 0.0], [3.0, 2.0, 1.0]])
    Nmc = 2000
    rq = O.OracleRequest(pts, Nmc=Nmc, kNStep=(20, 20, 20), xRange=(4.0, 4.0, 4.0))
    g = rq.geometry()
    kp, _, S = rq.kpoints()
    f = rq.generate()
    var_th = g.ampMult ** 2 / 2 * S.sum()
    assert f.var(axis=0).mean() == pytest.approx(var_th, rel=0.06)
    for lag, j in ((h, 1), (2 * h, 2)):
        cov_th = g.ampMult ** 2 / 2 * (S * np.cos(kp[:, 0] * lag)).sum()
        cov = np.mean(f[:, 0] * f[:, j])
        assert cov == pytest.approx(cov_th, abs=0.06 * var_th)
        # the left Riemann sum from k1 = 0 adds about dk/(2 pi) of constant
        assert cov_th / var_th == pytest.approx(math.exp(-PI * lag ** 2), abs=0.06)


def test_isotropic_unit_variance():
    pts = uniform_points(4, 5.0, seed=9)
    rq = O.OracleRequest(pts, Nmc=2000, method=O.ISOTROPIC, isoNRadial=64, isoNDir=16)
    kp, amp, S = rq.kpoints()
    f = rq.generate()
    var_th = (amp ** 2).sum() / 2
    # the radial sum stops at kMax = 7.355 (spectra_RF.f90:37), which holds
    # 96.7% of the 3-D spectral mass
    assert var_th == pytest.approx(0.9672, abs=0.002)
    assert f.var(axis=0).mean() == pytest.approx(var_th, rel=0.07)


# ------------------------------------------------- marginal, normalisation
def test_marginal_formulas():
    L = O.lib()
    z = np.linspace(-3, 3, 101)
    g = z.copy()
    assert L.rfo_marginal(O.FOM_GAUSSIAN, 2.0, 9.0, g.ctypes.data_as(C.POINTER(C.c_double)), g.size) == 0
    np.testing.assert_allclose(g, z * 3.0 + 2.0, rtol=1e-15)
    ln = z.copy()
    assert L.rfo_marginal(O.FOM_LOGNORMAL, 1.0, 0.25, ln.ctypes.data_as(C.POINTER(C.c_double)), ln.size) == 0
    s2 = math.log(1 + 0.25)
    np.testing.assert_allclose(ln, np.exp(z * math.sqrt(s2) + (math.log(1.0) - s2 / 2)), rtol=1e-15)
    bad = z.copy()
    assert L.rfo_marginal(O.FOM_LOGNORMAL, 0.0, 1.0, bad.ctypes.data_as(C.POINTER(C.c_double)), bad.size) != 0


def test_lognormal_moments_after_normalisation():
    x = uniform_points(20000, 10.0, seed=11)
    rq = O.OracleRequest(x, Nmc=2, kNStep=(6, 6, 6), margiFirst=O.FOM_LOGNORMAL, fieldAvg=1.0, fieldVar=0.25,
                         normalize=True)
    f = rq.generate()
    # exact: normalisation makes each column's log mean/variance exact
    s2 = math.log(1.25)
    lg = np.log(f)
    np.testing.assert_allclose(lg.mean(axis=1), -s2 / 2, atol=1e-12)
    np.testing.assert_allclose(lg.var(axis=1), s2, rtol=1e-10)


def test_normalize_literal_first_column_only():
    x = uniform_points(3000, 6.0, seed=2)
    f = O.OracleRequest(x, Nmc=3, kNStep=(5, 5, 5), normalize=True, literal=True).generate()
    assert abs(f[0].mean()) < 1e-12 and f[0].std() == pytest.approx(1.0, rel=1e-12)
    assert abs(f[1].std() - 1.0) > 1e-6


# ---------------------------------------------------- partition of unity
def test_unity_partition_cosine_taper():
    up = O.unity_partition([10, 7, 6], [3, 2, 0]).reshape(6, 7, 10)  # [z, y, x]
    N = 3
    w_hi = [(1 + math.cos(PI * s / (N + 2))) / 2 for s in range(1, N + 1)]
    np.testing.assert_allclose(up[0, 3, 7:10], w_hi, rtol=1e-15)
    np.testing.assert_allclose(up[0, 3, 0:3], w_hi[::-1], rtol=1e-15)
    assert np.all(up[:, 2:5, 3:7] == 1.0)
    assert np.all((up > 0) & (up <= 1))
    assert np.all(O.unity_partition([10, 7, 6], [3, 2, 0], faceMask=0) == 1.0)
    assert O.lib().rfo_overlap_npoints(0.5, 1.0, 0.05) == 9


# --------------------------------------------------------- CPU baseline
def test_baseline_matches_generate():
    x = grid(10, 0.15)
    rq = O.OracleRequest(x, Nmc=3, kNStep=(6, 6, 6))
    full = rq.generate()
    out, t = rq.baseline(100, 400, 1, 2, nthreads=2)
    assert t > 0
    np.testing.assert_allclose(out, full[1:3, 100:500], rtol=0, atol=1e-12)


# ------------------------------------------------------- randomization (3)
def test_randomization_wavevectors_are_the_first_draws():
    """Method 3 (gen_Std_Gauss_Randomization, randomFieldND.f90:343-361):
    kPoints_base = random_number * kMax (spectra_RF.f90:119-124), axis
    fastest, drawn before the phases, then the set_kSign copies."""
    x = grid(6, 0.2)
    rq = O.OracleRequest(x, Nmc=2, method=O.RANDOMIZATION, kNStep=(4, 3, 5), seedStart=3)
    g = rq.geometry()
    kn = 4 * 3 * 5
    assert g.K == 4 * kn
    kp, amp, S = rq.kpoints()
    r = O.rng(3)
    u = np.array([O.lib().rfo_rng_r8_uni_01(C.byref(r)) for _ in range(3 * kn)]).reshape(kn, 3)
    np.testing.assert_array_equal(kp[:kn], u * g.kMax)
    signs = [(1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1)]
    for q, sg in enumerate(signs):
        np.testing.assert_array_equal(kp[q * kn:(q + 1) * kn], u * g.kMax * np.array(sg))
    np.testing.assert_allclose(amp, np.sqrt(np.prod(np.exp(-kp ** 2 / (4 * 3.1415926535898)), axis=1)), rtol=1e-13)
    # the phases follow the 3*kn wavevector draws
    Bc, Bs = rq.phase_matrix()  # [r, k]
    phi0 = np.arctan2(-Bs[0], Bc[0])
    r = O.rng(3)
    for _ in range(3 * kn):
        O.lib().rfo_rng_i4_uni(C.byref(r))
    u0 = np.array([O.lib().rfo_rng_r8_uni_01(C.byref(r)) for _ in range(g.K)])
    ref = np.angle(np.exp(1j * 2 * 3.1415926535898 * u0))
    nz = amp > 1e-12
    np.testing.assert_allclose(np.angle(np.exp(1j * phi0[nz])), ref[nz], atol=1e-9)


def test_randomization_amplitude_unit_variance_and_literal_ampmult():
    """Intended: a random wavevector of a quadrant stands for kMax^D/kn of the
    spectral volume, so ampMult = 2 sqrt(kMax^D/(kn (2 pi)^D)) and the
    ensemble variance ampMult^2/2 * sum S is 1 (up to the kMax truncation and
    the Monte Carlo error of K random wavevectors).  Literal: the reference's
    2 sqrt(1/(K (2 pi)^D)) (randomFieldND.f90:262)."""
    x = grid(4, 0.3)
    PI = 3.1415926535898
    rq = O.OracleRequest(x, Nmc=1, method=O.RANDOMIZATION, kNStep=(16, 16, 16), seedStart=1)
    g = rq.geometry()
    kn = 16 ** 3
    assert math.isclose(g.ampMult, 2 * math.sqrt(g.kMax ** 3 / (kn * (2 * PI) ** 3)), rel_tol=1e-14)
    _, amp, S = rq.kpoints()
    var = g.ampMult ** 2 / 2 * S.sum()
    assert abs(var - 0.99) < 0.05, var
    lit = O.OracleRequest(x, Nmc=1, method=O.RANDOMIZATION, kNStep=(16, 16, 16), seedStart=1, literal=True)
    assert math.isclose(lit.geometry().ampMult, 2 * math.sqrt(1 / (4 * kn * (2 * PI) ** 3)), rel_tol=1e-14)
