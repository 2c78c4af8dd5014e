"""The fixed-point phase of the table generator (rf_gen.cuh::table_pairs_fxp,
tables written by rf_tables.cu::table_element), restated in numpy and
checked against the exact phase k.x on the CPU.

Per component: x = A/4 + b with integer A and |b| <= 1/8; k/2pi = C 2^-30 + e
with integer C; the coarse phase is the wrapped 32-bit integer dot product
sum A_d C_d (units of 2^-32 turn), truncated to 2^-23 turn; the fine phase
sum b_d k_d is FP32 (fused multiply-adds) with half a unit added so that the
truncation rounds.  For points with |x|_1 <= 128 correlation lengths the
angle handed to the SFU is within 1e-6 rad of k.x modulo 2 pi (the dropped
term is below |x|_1 2^-31 turn) and within [-1.51 pi, 1.51 pi] for the
isotropic wavevectors (|k| <= kMax = 7.355).  float32 fused multiply-adds are
emulated in float64 (exact products) with one final rounding.
"""
import numpy as np

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
