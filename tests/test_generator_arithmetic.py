"""The trig-tile generators' arithmetic (rf_gen.cuh), restated in numpy and
checked against exact phases on the CPU:

- the fixed-point phase of the table generator (table_pairs_fxp, tables
  written by rf_tables.cu::table_element).  Per component x = A/4 + b with
  integer A and |b| <= 1/8, k/2pi = C 2^-30 + e with integer C; the coarse
  phase is the wrapped 32-bit integer dot product sum A_d C_d (units of
  2^-32 turn) truncated to 2^-23 turn, the fine phase sum b_d k_d is FP32
  (fused multiply-adds) with half a unit added so that the truncation
  rounds.  For points with |x|_1 <= 128 correlation lengths the angle is
  within 1e-6 rad of k.x modulo 2 pi and within [-1.51 pi, 1.51 pi] for the
  isotropic wavevectors (|k| <= kMax = 7.355);
- the FP64 reduction of the table generator's FAST form (table_pairs<true>);
- the outer-phasor walk of GEN_GRID3 (Grid3Walk);
- the outer-group factorisation of GEN_OUTER (rf_outer.cu, and the operand
  rf_tables.cu outer_element writes), against the oracle's field.
float32 fused multiply-adds are emulated in float64 (exact products) with
one final rounding.
"""
import numpy as np

from oracle import oracle as O

UNIT = np.float32(6.283185307179586) * np.float32(2.0 ** -23)  # radians per 2^-23 turn


def fmaf(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def fxp_angle(x, k):
    """x: (n, 3) FP64 points; k: (m, 3) FP64 wavevectors -> (n, m) angles."""
    t = k / 6.283185307179586  # turns, as the table builder writes them
    C = np.rint(t * 2.0 ** 30).astype(np.int64).astype(np.uint32)
    kf = k.astype(np.float32)
    A = np.rint(x * 4.0)
    b = (x - 0.25 * A).astype(np.float32)
    A = A.astype(np.int64).astype(np.uint32)
    P = np.zeros((x.shape[0], k.shape[0]), dtype=np.uint32)
    s = np.full(P.shape, np.float32(0.5) * UNIT, dtype=np.float32)
    for d in range(3):
        P = P + A[:, d:d + 1] * C[None, :, d]  # uint32 arithmetic wraps
        s = fmaf(b[:, d:d + 1], kf[None, :, d], s)
    q = P.view(np.int32) >> 9
    qf = q.astype(np.float32)  # |q| < 2^22: exact
    return fmaf(qf, np.broadcast_to(UNIT, qf.shape), s)


def test_fixed_point_phase_error_bound():
    rs = np.random.RandomState(5)
    n, m = 4000, 256
    # points spread over |x|_1 <= 128, wavevectors |k| <= kMax (isotropic) and grid-like ones
    x = rs.uniform(-1, 1, size=(n, 3))
    x *= (128.0 * rs.uniform(0, 1, size=(n, 1)) ** 0.5) / np.abs(x).sum(axis=1, keepdims=True)
    kdir = rs.normal(size=(m, 3))
    k = kdir / np.linalg.norm(kdir, axis=1, keepdims=True) * rs.uniform(0, 7.355, size=(m, 1))
    r = fxp_angle(x, k).astype(np.float64)
    exact = (x.astype(np.longdouble) @ k.astype(np.longdouble).T)
    two_pi = 2 * np.pi
    d = np.asarray((r - exact) % two_pi, dtype=np.float64)
    d = np.where(d > np.pi, d - two_pi, d)
    assert np.abs(d).max() <= 1e-6
    assert np.sqrt(np.mean(d ** 2)) <= 3e-7
    assert np.abs(r).max() <= 1.51 * np.pi


def test_fixed_point_phase_wraps_exactly_far_from_the_origin():
    """The coarse term is exact modulo one turn at any magnitude: shifting a
    point by a whole number of periods of every wavevector's grid leaves the
    integer part's contribution unchanged modulo 2^32."""
    k = np.array([[0.5, -1.25, 2.0], [7.0, 0.0, -3.5]])
    x = np.array([[0.1, 0.2, -0.3], [60.0, -40.0, 27.75]])
    r = fxp_angle(x, k).astype(np.float64)
    exact = (x @ k.T) % (2 * np.pi)
    d = (r - exact) % (2 * np.pi)
    d = np.where(d > np.pi, d - 2 * np.pi, d)
    assert np.abs(d).max() <= 1e-6


def test_fast_fp64_reduction_of_the_table_phase():
    """table_pairs<FAST>: the phase in turns plus 1.5 * 2^20 (+ half a unit of
    2^-23) puts it on the FP64 grid of 2^-32 turn, so the sum's low word is
    the phase modulo one turn in 32-bit fixed point; an arithmetic shift keeps
    2^-23 turn.  The angle stays within 2^-24 turn of the FP64 phase (plus the
    FP32 product's rounding) and inside [-pi, pi], for |x.k| < 2^18 turns."""
    rs = np.random.RandomState(9)
    th = np.concatenate([rs.uniform(-1, 1, 20000) * 2.0 ** e for e in (0, 4, 10, 17)])  # turns
    shift = 1572864.0 + 2.0 ** -24
    low = (np.asarray(th + shift, dtype=np.float64).view(np.uint64) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    q = low.view(np.int32) >> 9
    r = q.astype(np.float32) * UNIT  # the float through 0x4B400000 + q equals q exactly
    exact = 2 * np.pi * (th - np.rint(th))
    d = r.astype(np.float64) - exact
    d = (d + np.pi) % (2 * np.pi) - np.pi
    assert np.abs(d).max() <= 2 * np.pi * 2.0 ** -24 + 4e-7
    assert np.abs(r).max() <= np.pi * (1 + 2.0 ** -20)


def test_grid3_outer_phasor_walk():
    """GEN_GRID3's E1(i1) = E1(i1 - 1) E1(1) in FP32 complex products from
    E1(0) = 1, restarted at every wrap (at most 31 products): relative error
    below 4e-6 of the exact exp(i i1 k1 x1)."""
    rs = np.random.RandomState(11)
    theta = rs.uniform(-np.pi, np.pi, 5000)  # k1(1) x1 reduced, as axis_phasor returns it
    c, s = np.cos(theta).astype(np.float32), np.sin(theta).astype(np.float32)
    er, ei = np.ones_like(c), np.zeros_like(c)
    worst = 0.0
    for i in range(1, 32):
        er, ei = er * c - ei * s, er * s + ei * c  # float32 arithmetic
        ex = np.exp(1j * i * theta)
        worst = max(worst, float(np.abs((er.astype(np.float64) + 1j * ei.astype(np.float64)) - ex).max()))
    assert worst <= 4e-6


def test_outer_group_factorisation_equals_oracle():
    """The outer-group contraction of rf_outer.cu restated in numpy: A = the
    outer phasors (Re, Im of E1(i1) E2(i2)^{s2}), B = the four coefficients
    built from the s3 = +/- pair of each (outer group, i3) exactly as
    rf_tables.cu outer_element writes them, and the epilogue's sum over i3
    with cos and sin of k3 x3.  Equals the oracle's point-by-point sum."""
    x = O.grid([0.0, 0.0, 0.0], [0.13, 0.11, 0.17], [7, 6, 5])
    kn, Nmc = (5, 4, 3), 3
    req = O.OracleRequest(x, Nmc=Nmc, kNStep=kn)
    ref = req.generate()
    g = req.geometry()
    Bc, Bs = req.phase_matrix()  # [r, k]: a cos(phi), -a sin(phi)
    n1, n2, n3 = kn
    n123 = n1 * n2 * n3
    f = np.zeros_like(ref)
    for s2 in range(2):
        for i2 in range(n2):
            for i1 in range(n1):
                k2 = g.kDelta[1] * i2 * (-1.0 if s2 else 1.0)
                P = np.exp(1j * (g.kDelta[0] * i1 * x[:, 0] + k2 * x[:, 1]))
                for i3 in range(n3):
                    kp = 2 * s2 * n123 + i1 + n1 * (i2 + n2 * i3)
                    km = kp + n123
                    W = (Bc[:, kp] + Bc[:, km], Bs[:, kp] + Bs[:, km], Bs[:, kp] - Bs[:, km], Bc[:, km] - Bc[:, kp])
                    c3, s3 = np.cos(g.kDelta[2] * i3 * x[:, 2]), np.sin(g.kDelta[2] * i3 * x[:, 2])
                    f += (np.outer(W[0], P.real * c3) + np.outer(W[1], P.imag * c3) + np.outer(W[2], P.real * s3)
                          + np.outer(W[3], P.imag * s3))
    f *= g.ampMult
    assert np.abs(f - ref).max() <= 1e-12 * np.abs(ref).max()


def _bf16(a):
    """Round to BF16 (nearest even), returned as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _tf32(a):
    """Round to TF32 (10 mantissa bits, nearest, ties away from zero: half a
    unit added to the magnitude bits, the low 13 bits cleared), as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x1000) & 0xFFFFE000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _outer_sample():
    """The 128^3 workload's outer-group operands on a sample of 96 point
    columns x 128 points: (A, W, the K-step variance weights, field(a, b),
    the exact field, K-step mask -> K-element mask)."""
    n1 = n2 = n3 = 24
    Nmc, corrL, h, N = 64, (2.0, 1.0, 0.5), 0.05, 128
    req = O.OracleRequest(np.zeros((1, 3)), Nmc=Nmc, kNStep=(24, 24, 24), corrL=corrL, xRange=((N - 1) * h,) * 3)
    g = req.geometry()
    Bc, Bs = req.phase_matrix()
    kd, n123, G = list(g.kDelta), n1 * n2 * n3, 2 * n1 * n2
    W = np.zeros((G, 2, n3, 2, Nmc))
    i3 = np.arange(n3)
    for s2 in range(2):
        for i2 in range(n2):
            for i1 in range(n1):
                gg = i1 + n1 * (i2 + n2 * s2)
                kp = 2 * s2 * n123 + i1 + n1 * (i2 + n2 * i3)
                km = kp + n123
                bcP, bsP, bcM, bsM = Bc[:, kp].T, Bs[:, kp].T, Bc[:, km].T, Bs[:, km].T
                W[gg, 0, :, 0], W[gg, 1, :, 0] = bcP + bcM, bsP + bsM
                W[gg, 0, :, 1], W[gg, 1, :, 1] = bsP - bsM, bcM - bcP
    W = W.reshape(2 * G, 2 * n3 * Nmc)
    # K-step j = i2 + n2 (s2 + 2 jj) holds the groups i1 = 8 jj .. 8 jj + 7 (rf_plan.h outer_kstep)
    pi_ref = 3.1415926535898
    w = np.array([np.exp(-(kd[0] * np.arange(8 * (j // (2 * n2)), 8 * (j // (2 * n2)) + 8)) ** 2 / (4 * pi_ref)).sum()
                  * np.exp(-(kd[1] * (j % n2)) ** 2 / (4 * pi_ref)) for j in range(3 * n2 * 2)])

    def kmask(lo):
        g_lo = np.array([lo[i2 + n2 * (s2 + 2 * (i1 // 8))] for s2 in range(2) for i2 in range(n2)
                         for i1 in range(n1)])
        return np.repeat(g_lo, 2)

    rs = np.random.RandomState(3)
    J1, J2 = rs.randint(0, N, 96), rs.randint(0, N, 96)
    x = np.arange(N) * h
    A = np.zeros((96, 2 * G))
    for s2 in range(2):
        P = np.exp(1j * (kd[0] * np.arange(n1)[None, None, :] * (x[J1] / corrL[0])[:, None, None]
                         + (-1 if s2 else 1) * kd[1] * np.arange(n2)[None, :, None] * (x[J2] / corrL[1])[:, None, None]))
        gi = (np.arange(n1)[None, :] + n1 * (np.arange(n2)[:, None] + n2 * s2)).ravel()
        A[:, 2 * gi], A[:, 2 * gi + 1] = P.reshape(96, -1).real, P.reshape(96, -1).imag
    E3 = np.exp(1j * kd[2] * i3[None, :] * (x / corrL[2])[:, None])  # [j3, i3]

    def field(a, b):
        Y = (a @ b).reshape(96, n3, 2, Nmc)
        return (np.einsum('ji,pir->pjr', E3.real, Y[:, :, 0])
                + np.einsum('ji,pir->pjr', E3.imag, Y[:, :, 1])).reshape(-1, Nmc)

    return A, W, w, field, field(A, W), kmask


def _variance_mask(w, left):
    """The K-steps carrying all but `left` of the variance, ranked as
    rf_host.cu outer_rank_masks ranks them."""
    lo = np.zeros(w.size, bool)
    cov = 0.0
    for j in sorted(range(w.size), key=lambda j: (-w[j], j)):
        lo[j] = cov < (1.0 - left) * w.sum()
        cov += w[j]
    return lo


def _errors(f, exact):
    rel = np.sqrt(((f - exact) ** 2).sum() / (exact ** 2).sum())
    per = np.sqrt(((f - exact) ** 2).sum(0) / (exact ** 2).sum(0))
    return rel, per.max()


def test_outer_group_bf16_error_budget():
    """A BF16 hi/lo split of the outer-group operands (the alternative the
    TF32 K-steps of rf_outer.cu are measured against) emulated on the 128^3
    workload (24^3 x 4 wavevectors, corrL (2, 1, 0.5), Nmc 64) on a
    sample of 96 point columns x 128 points: A = the outer phasors and W = the
    coefficients rounded to BF16, each with its lo term (the rounding residual,
    rounded again) on the K-steps that carry all but 30 % of the field variance,
    ranked as rf_host.cu outer_rank_masks ranks them; the epilogue's i3 sum
    exact.
    Without lo terms the relative L2 error is about 2.1e-3 (above the 2e-3
    bound); with them it is about 1.2e-3, the worst realization under 1.5e-3."""
    A, W, w, field, exact, kmask = _outer_sample()
    k_lo = kmask(_variance_mask(w, 0.3))
    Ah, Wh = _bf16(A), _bf16(W)
    none = field(Ah, Wh)
    split = field(Ah + np.where(k_lo[None, :], _bf16(A - Ah), 0.0), Wh + np.where(k_lo[:, None], _bf16(W - Wh), 0.0))
    assert _errors(none, exact)[0] > 2e-3
    rel, worst = _errors(split, exact)
    assert rel < 1.3e-3 and worst < 1.5e-3, (rel, worst)


def test_outer_group_tf32_error_budget():
    """The BF16 outer-group plans (rf_outer.cu, rf_outer_pair.cu, oTf32):
    the K-steps carrying all but 25 % of the variance take A and W rounded to TF32 (two
    kind::tf32 MMAs of K = 8, the values rounded by tf32_bits as the generators
    and rf_tables.cu outer_run round them), the others A and W rounded to BF16
    alone.  Relative L2 about 1.08e-3, worst realization about 1.17e-3: below
    the BF16 hi/lo form at 0.3 (1.16e-3, 1.30e-3), at 1.26x the MMA cycles of
    the BF16 hi terms alone against 1.46x."""
    A, W, w, field, exact, kmask = _outer_sample()
    lo = _variance_mask(w, 0.25)
    k_tf = kmask(lo)
    mixed = field(np.where(k_tf[None, :], _tf32(A), _bf16(A)), np.where(k_tf[:, None], _tf32(W), _bf16(W)))
    rel, worst = _errors(mixed, exact)
    assert rel < 1.12e-3 and worst < 1.22e-3, (rel, worst)
    cycles = (lo.size - lo.sum()) + 2 * lo.sum()  # BF16 K-step: one MMA per half; TF32: two of the same length
    assert cycles / lo.size < 1.3
    # the rounding is the nearest TF32 value, ties away from zero
    v = np.array([1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, -(1.0 + 2.0 ** -11), 1.0 + 2.0 ** -12], np.float32)
    assert list(_tf32(v)) == [1.0 + 2.0 ** -10, 1.0 + 2 * 2.0 ** -10, -(1.0 + 2.0 ** -10), 1.0]
