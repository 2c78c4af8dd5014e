"""Caller-supplied uniform draws (rf_options.draws) in place of rnglib.

With draws equal to rnglib's own stream (the oracle's sequential i4_uni
values times 4.656613057e-10, rnglib.f90:1517) every method must give the
field of the default path bit for bit: that pins the position of every draw
(Shinozuka phases, randomization base wavevectors, isotropic directions,
gamma and psi blocks).  With arbitrary draws the field must be the
Shinozuka sum f = ampMult sum_k a_k cos(k.x + 2 pi U[r K + k])
(randomFieldND.f90:276-330) evaluated in FP64 from the oracle's wavevectors
and amplitudes.
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.helpers import errors, grid, uniform_points

R8 = 4.656613057e-10


def _stream(seed, count):
    return O.i4_stream(seed, count).astype(np.float64) * R8


def test_draws_rejected_where_not_taken():
    """Entry points without caller draws refuse them in validation, before
    any device work (the buffer addresses are never used)."""
    x = grid(4, 0.1)
    with pytest.raises(rf.RandomFieldError) as e:
        rf.generate_device_noalloc(256, 3, x.shape[0], 1, 1, [1.0] * 3, 0.0, 1.0, 2, rf.SHINOZUKA, 256,
                                   k_nstep=(4, 4, 4), draws=np.zeros(16))
    assert e.value.code == -10  # RF_ENOTSUP


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["bf16", "fp32", "fp16"])
def test_shinozuka_stream_draws_equal_default(prec):
    x = grid(16, 0.1)
    kn, Nmc, seed = (12, 12, 12), 5, 3
    a = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", [1.0] * 3, 0.0, 1.0, Nmc,
                                                   rf.SHINOZUKA, precision=prec, k_nstep=kn, seed_start=seed)
    K = 4 * int(np.prod(kn))
    b = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", [1.0] * 3, 0.0, 1.0, Nmc,
                                                   rf.SHINOZUKA, precision=prec, k_nstep=kn, seed_start=99,
                                                   draws=_stream(seed, Nmc * K))
    assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.gpu
@pytest.mark.parametrize("method,nDim,opts", [
    (rf.ISOTROPIC, 3, dict(iso_n_radial=12, iso_n_dir=10)),
    (rf.ISOTROPIC, 2, dict(iso_n_radial=12, iso_n_dir=10)),
    (rf.RANDOMIZATION, 3, dict(k_nstep=(6, 5, 4))),
])
def test_other_methods_stream_draws_equal_default(method, nDim, opts):
    x = uniform_points(3000, 5.0, nDim=nDim, seed=4)
    Nmc, seed = 4, 7
    corrL = [1.0] * nDim
    a = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", corrL, 0.0, 1.0, Nmc, method,
                                                   precision="fp32", seed_start=seed, **opts)
    K = rf.query_geometry(x.T, "gaussian", corrL, method, **opts)[0]
    if method == rf.ISOTROPIC:
        need = (2 if nDim == 3 else 1) * K + Nmc * 2 * K
    else:
        need = (K >> (nDim - 1)) * nDim + Nmc * K
    b = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", corrL, 0.0, 1.0, Nmc, method,
                                                   precision="fp32", seed_start=99, draws=_stream(seed, need),
                                                   **opts)
    assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp32", None), ("bf16", 2e-3)])
def test_arbitrary_draws_give_the_shinozuka_sum(prec, tol):
    x = grid(8, 0.13)
    kn, Nmc = (6, 5, 4), 3
    K = 4 * int(np.prod(kn))
    U = np.random.RandomState(11).uniform(0.0, 1.0, Nmc * K)
    got = np.asarray(rf.create_standard_gaussian_field_unstruct(
        x.T, "gaussian", "gaussian", [1.0] * 3, 0.0, 1.0, Nmc, rf.SHINOZUKA, precision=prec, k_nstep=kn,
        draws=U)).T
    rq = O.OracleRequest(x, Nmc=Nmc, kNStep=kn)
    kp, amp, _ = rq.kpoints()
    g = rq.geometry()
    phase = x @ kp.T  # [i, k]
    ref = np.stack([g.ampMult * (np.cos(phase + 2.0 * 3.1415926535898 * U[r * K:(r + 1) * K]) @ amp)
                    for r in range(Nmc)])
    if tol is None:
        assert errors(got, ref)[0] <= 1e-5 * ref.std(), errors(got, ref)
    else:
        assert errors(got, ref)[1] <= tol, errors(got, ref)


@pytest.mark.gpu
def test_too_few_draws_rejected():
    x = grid(4, 0.1)
    with pytest.raises(rf.RandomFieldError) as e:
        rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", [1.0] * 3, 0.0, 1.0, 2,
                                                   rf.SHINOZUKA, k_nstep=(4, 4, 4), draws=np.zeros(10))
    assert e.value.code == -9 and "draws" in str(e.value)
