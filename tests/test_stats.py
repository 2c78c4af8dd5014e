"""Field statistics (statistics_RF.f90): the oracle's restatement and the
device entry point rf_field_statistics.

CPU: the oracle's FFT route (rebuild_Sk_FFT's forward FFT / N, times the
conjugate, mean over the lines, unnormalised backward FFT) equals the direct
circular autocorrelation the device sums, and a single cosine mode gives its
known correlation cos(2 pi k0 l / N) exactly.
GPU: on a field generated on the device, the moments, the lags and the
correlation lengths equal the oracle's on the same field (FP64, different
summation order: relative 1e-12 for moments, absolute 1e-12 for lags);
repeated calls are bitwise equal; the lags of a large grid follow the target
correlation exp(-pi (r/L)^2) up to 3 L (statistical bound 0.08); bad grids
are refused.
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O


@pytest.mark.parametrize("shape", [(32,), (16, 12), (12, 10, 8)])
def test_oracle_fft_route_equals_direct_sum(shape):
    rs = np.random.RandomState(3)
    n = int(np.prod(shape))
    f = rs.normal(size=(n, 2)) * 1.7 + 0.3
    st = O.field_statistics(f, shape, [0.1] * len(shape))
    g = (f[:, 0] - st["global_avg"]) / st["global_std"]
    direct = O.circular_autocorrelation(g, shape)
    for a, b in zip(st["sk"], direct):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
    np.testing.assert_allclose(st["evnt_avg"], f.mean(axis=0), rtol=1e-13)
    np.testing.assert_allclose(st["evnt_std"], f.std(axis=0), rtol=1e-12)


def test_oracle_single_mode_known_answer():
    N, k0 = 64, 5
    z = np.arange(N)
    f = np.cos(2 * np.pi * k0 * z / N)[:, None]
    st = O.field_statistics(f, (N,), (0.5,))
    np.testing.assert_allclose(st["sk"][0], np.cos(2 * np.pi * k0 * np.arange(N // 2) / N), atol=1e-12)
    R = st["sk"][0]
    assert st["corrL"][0] == pytest.approx(2.0 * (R.sum() - (R[0] + R[-1]) / 2.0) * 0.5)


# ---------------------------------------------------------------- GPU
def _grid(shape, h):
    return O.grid([0.0] * len(shape), [h] * len(shape), list(shape))


@pytest.fixture(scope="module")
def ctx():
    c = rf.Context(0)
    yield c
    c.close()


def _device_field(ctx, pts, Nmc, prec, **opts):
    torch = pytest.importorskip("torch")
    n, nDim = pts.shape
    dx = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    dout = torch.empty((Nmc, n), dtype=torch.float64, device="cuda")
    ctx.generate(dx, nDim, n, 1, 1, (1.0,) * nDim, 0.0, 1.0, Nmc, 2, dout, precision=prec, **opts)
    ctx.synchronize()
    return dout


@pytest.mark.gpu
@pytest.mark.parametrize("shape,prec", [((40, 36, 32), "bf16"), ((48, 40), "fp32"), ((300,), "fp16")])
def test_device_statistics_match_oracle(ctx, shape, prec):
    h = 0.15
    pts = _grid(shape, h)
    Nmc = 3
    kn = {3: (16, 16, 16), 2: (24, 24, 0), 1: (64, 0, 0)}[len(shape)]
    dout = _device_field(ctx, pts, Nmc, prec, k_nstep=kn, seed_start=11)
    n = pts.shape[0]
    got = ctx.field_statistics(dout, n, Nmc, len(shape), grid=shape, step=[h] * len(shape))
    field = dout.cpu().numpy().T  # n x Nmc
    ref = O.field_statistics(field, shape, [h] * len(shape))
    sd = ref["global_std"]
    np.testing.assert_allclose(got["evnt_avg"], ref["evnt_avg"], rtol=0, atol=1e-12 * sd)
    np.testing.assert_allclose(got["evnt_std"], ref["evnt_std"], rtol=1e-12)
    assert got["global_avg"] == pytest.approx(ref["global_avg"], abs=1e-12 * sd)
    assert got["global_std"] == pytest.approx(ref["global_std"], rel=1e-12)
    for a, b in zip(got["sk"], ref["sk"]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
    np.testing.assert_allclose(got["corrL"], ref["corrL"], rtol=1e-10)
    again = ctx.field_statistics(dout, n, Nmc, len(shape), grid=shape, step=[h] * len(shape))
    for a, b in zip(got["sk"], again["sk"]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(got["evnt_std"], again["evnt_std"])


@pytest.mark.gpu
def test_moments_of_unstructured_points(ctx):
    rs = np.random.RandomState(4)
    pts = rs.uniform(0.0, 6.0, size=(5000, 3))
    dout = _device_field(ctx, pts, 5, "bf16", k_nstep=(16, 16, 16))
    got = ctx.field_statistics(dout, 5000, 5, 3)
    ref = O.field_statistics(dout.cpu().numpy().T)
    np.testing.assert_allclose(got["evnt_std"], ref["evnt_std"], rtol=1e-12)
    assert "sk" not in got


@pytest.mark.gpu
def test_lags_follow_the_target_correlation(ctx):
    # 96^3 points 0.2 apart: 19 correlation lengths per axis (the 24-point
    # wavenumber grid repeats after 2 pi / kDelta = 19.6)
    shape, h = (96, 96, 96), 0.2
    pts = _grid(shape, h)
    dout = _device_field(ctx, pts, 1, "bf16", k_nstep=(24, 24, 24), seed_start=3)
    got = ctx.field_statistics(dout, pts.shape[0], 1, 3, grid=shape, step=[h] * 3)
    lags = np.arange(16) * h  # up to 3 L
    target = np.exp(-np.pi * lags ** 2)
    # rebuild_corrL integrates all N/2 lags: on a line of 19 L the lags beyond
    # 3 L sit on the variance of the line means (about 0.05), so its estimate
    # of L is biased up here; it is checked against the oracle above, and
    # the lags themselves against the target here
    for d in range(3):
        assert np.abs(got["sk"][d][:16] - target).max() < 0.08, (d, got["sk"][d][:16])


@pytest.mark.gpu
def test_bad_grids_are_refused(ctx):
    torch = pytest.importorskip("torch")
    d = torch.zeros((1, 100), dtype=torch.float64, device="cuda")
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.field_statistics(d, 100, 1, 2, grid=(10, 11), step=(1.0, 1.0))
    assert e.value.code == -9
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.field_statistics(d, 100, 1, 2, grid=(100, 1), step=(1.0, 1.0))
    assert e.value.code == -9
    big = torch.zeros((1, 5000), dtype=torch.float64, device="cuda")
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.field_statistics(big, 5000, 1, 1, grid=(5000,), step=(1.0,))
    assert e.value.code == -10
