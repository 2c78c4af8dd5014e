"""The FFT method (method 4, gen_Std_Gauss_FFT): the oracle's restatement and
the device entry point rf_generate_fft_grid.

CPU: scipy's DCT type 3 (the oracle's route) is FFTW's REDFT01, checked
against the defining sum Y_i = X_0 + 2 sum_{j>=1} X_j cos(pi j (2i+1)/(2n))
on a small grid and on two known answers; the draws follow the reference's
order (K gamma draws, K - 1 skipped, K phi draws).
GPU: the device field equals the oracle's on the same grid and seed (both
FP64: relative-L2 <= 1e-11), in 2-D and 3-D, both marginals, cm_COS, with
realization r drawn from seed_start + r; invalid grids are refused.
"""
import itertools

import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O


def _dct3_direct(X):
    """Separable DCT-III by its defining sum (FFTW REDFT01), every axis."""
    Y = np.asarray(X, dtype=np.float64)
    for ax in range(Y.ndim):
        n = Y.shape[ax]
        i = np.arange(n)[:, None]
        j = np.arange(n)[None, :]
        C = np.where(j == 0, 1.0, 2.0 * np.cos(np.pi * j * (2 * i + 1) / (2 * n)))
        Y = np.moveaxis(np.tensordot(C, np.moveaxis(Y, ax, 0), axes=(1, 0)), 0, ax)
    return Y


def test_scipy_dct3_is_redft01():
    from scipy import fft as sfft

    rs = np.random.RandomState(1)
    X = rs.normal(size=(5, 7, 6))
    np.testing.assert_allclose(sfft.dctn(X, type=3, norm=None), _dct3_direct(X), rtol=0, atol=1e-12)
    e0 = np.zeros(9)
    e0[0] = 1.0
    np.testing.assert_allclose(sfft.dct(e0, type=3, norm=None), np.ones(9), atol=1e-15)
    e1 = np.zeros(9)
    e1[1] = 1.0
    np.testing.assert_allclose(sfft.dct(e1, type=3, norm=None), 2 * np.cos(np.pi * (2 * np.arange(9) + 1) / 18),
                               atol=1e-15)


def test_oracle_draw_order_and_amplitudes():
    n, h, L = (6, 5), (0.2, 0.3), (1.0, 2.0)
    f = O.fft_method_field(n, h, L, seedStart=3)
    # restate the amplitudes from the raw stream and transform directly
    K = 30
    r = O.rng(3)
    u = [O.lib().rfo_rng_r8_uni_01(__import__("ctypes").byref(r)) for _ in range(3 * K - 1)]
    hn = np.array(h) / np.array(L)
    kd = 2 * O.PI_REF / (1.1 * (np.array(n) - 1) * hn)
    X = np.zeros((n[1], n[0]))
    for j, (i2, i1) in enumerate(itertools.product(range(n[1]), range(n[0]))):
        k1, k2 = i1 * kd[0], i2 * kd[1]
        S = np.exp(-k1 * k1 / (4 * O.PI_REF)) * np.exp(-k2 * k2 / (4 * O.PI_REF))
        X[i2, i1] = (u[j] - 0.5) * np.sqrt(S) * np.cos(2 * O.PI_REF * u[2 * K - 1 + j])
    ref = _dct3_direct(X).reshape(-1) * np.sqrt(np.prod(hn))
    np.testing.assert_allclose(f, ref, rtol=0, atol=1e-13 * np.abs(ref).max())


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def ctx():
    c = rf.Context(0)
    yield c
    c.close()


def _marginal(g, marg, avg, var):
    if marg == "gaussian":
        return g * np.sqrt(var) + avg
    nv = np.log(1 + var / avg ** 2)
    return np.exp(g * np.sqrt(nv) + np.log(avg) - nv / 2)


@pytest.mark.gpu
@pytest.mark.parametrize("n,h,L,marg,cm", [
    ((48, 40), (0.1, 0.15), (1.0, 2.0), "gaussian", "gaussian"),
    ((24, 20, 16), (0.2, 0.2, 0.1), (1.0, 1.0, 0.5), "lognormal", "gaussian"),
    ((17, 13, 9), (0.3, 0.3, 0.3), (1.0, 1.0, 1.0), "gaussian", "cos"),
])
def test_device_fft_method_matches_oracle(ctx, n, h, L, marg, cm):
    torch = pytest.importorskip("torch")
    K = int(np.prod(n))
    Nmc = 2
    avg, var = (1.0, 0.25) if marg == "lognormal" else (0.0, 1.0)
    d = torch.empty((Nmc, K), dtype=torch.float64, device="cuda")
    ctx.generate_fft_grid(d, n, h, cm, marg, L, avg, var, Nmc, seed_start=5)
    got = d.cpu().numpy()
    for r in range(Nmc):
        g = O.fft_method_field(n, h, L, seedStart=5 + r, corrMod=O.CM_COS if cm == "cos" else O.CM_GAUSSIAN)
        ref = _marginal(g, marg, avg, var)
        assert np.linalg.norm(got[r] - ref) <= 1e-11 * np.linalg.norm(ref), r
    again = torch.empty_like(d)
    ctx.generate_fft_grid(again, n, h, cm, marg, L, avg, var, Nmc, seed_start=5)
    np.testing.assert_array_equal(again.cpu().numpy(), got)


@pytest.mark.gpu
def test_fft_method_refuses_bad_grids(ctx):
    torch = pytest.importorskip("torch")
    d = torch.empty((1, 4096), dtype=torch.float64, device="cuda")
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.generate_fft_grid(d, (4096,), (0.1,), "gaussian", "gaussian", (1.0,), 0.0, 1.0, 1)
    assert e.value.code == -2  # 1-D: the reference stops
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.generate_fft_grid(d, (1, 4096), (0.1, 0.1), "gaussian", "gaussian", (1.0, 1.0), 0.0, 1.0, 1)
    assert e.value.code == -9
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.generate_fft_grid(d, (64, 64), (0.1, 0.0), "gaussian", "gaussian", (1.0, 1.0), 0.0, 1.0, 1)
    assert e.value.code == -9
