"""The device table builder's rnglib draws, bit for bit against a sequential
rnglib run.

The builder (randomfield_b200/csrc/rf_tables.cu) evaluates generator 1 of
rnglib (RANDLIB/rnglib.f90:548-659) by jump-ahead and stepping; here every
draw it consumed for a (realization, wavevector) is exported through
rf_debug_table_draws (the same runs, cursors and positions as the operand
build) and compared with the oracle's sequential stream, one i4_uni call
after another (oracle/rf_oracle.c rfo_rng_i4_uni, pinned on the L'Ecuyer-Cote
recurrences in tests/test_oracle.py).  Draw order of the reference:
  - Shinozuka: K phases per realization in k order (randomFieldND.f90:278-279);
  - randomization: the nDim * kn base-wavevector draws first
    (spectra_RF.f90:119-124), then the phases;
  - isotropic: the phi and theta direction blocks, then per realization a
    gamma block and a psi block (randomFieldND.f90:460-468 restated).
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SEEDS = [0, 1, 12345]


@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("prec", ["bf16", "fp32"])
def test_shinozuka_3d_grid_draws(seed, prec):
    # the 128^3 workload's wavevector grid: 24^3 x 4 = 55,296 (GEN_GRID3 kernel
    # order); 130 realizations: two realization blocks of the BF16 form
    Nmc = 130
    draws, _ = rf.debug_table_draws(3, rf.SHINOZUKA, Nmc, precision=prec, seed_start=seed, k_nstep=(24, 24, 24))
    K = draws.shape[1]
    assert K == 55296
    ref = O.i4_stream(seed, Nmc * K).reshape(Nmc, K)
    assert np.array_equal(draws, ref), int((draws != ref).sum())


@pytest.mark.parametrize("seed", SEEDS)
def test_shinozuka_2d_table_draws(seed):
    # 2-D: the explicit wavevector table (GEN_TABLE order = reference order),
    # K = 37 x 29 x 2 = 2146, not a multiple of the 32-wavevector runs
    Nmc = 70
    draws, _ = rf.debug_table_draws(2, rf.SHINOZUKA, Nmc, precision="fp16", seed_start=seed, k_nstep=(37, 29, 0))
    K = draws.shape[1]
    assert K == 37 * 29 * 2
    ref = O.i4_stream(seed, Nmc * K).reshape(Nmc, K)
    assert np.array_equal(draws, ref)


@pytest.mark.parametrize("seed", SEEDS)
def test_randomization_draws(seed):
    Nmc = 9
    kn = (11, 7, 5)
    draws, _ = rf.debug_table_draws(3, rf.RANDOMIZATION, Nmc, precision="bf16", seed_start=seed, k_nstep=kn)
    K = draws.shape[1]
    assert K == 4 * int(np.prod(kn))
    skip = int(np.prod(kn)) * 3  # nDim * kn base-wavevector draws come first
    ref = O.i4_stream(seed, skip + Nmc * K)[skip:].reshape(Nmc, K)
    assert np.array_equal(draws, ref)


@pytest.mark.parametrize("seed", SEEDS)
@pytest.mark.parametrize("nDim", [2, 3])
def test_isotropic_draws(seed, nDim):
    Nmc = 33
    draws, kd = rf.debug_table_draws(nDim, rf.ISOTROPIC, Nmc, precision="bf16", seed_start=seed, iso_n_radial=21,
                                     iso_n_dir=13)
    K = draws.shape[1]
    assert K == 21 * 13
    nblk = 2 if nDim == 3 else 1  # direction blocks: phi (3-D only), theta
    s = O.i4_stream(seed, nblk * K + Nmc * 2 * K)
    dirs = s[:nblk * K].reshape(nblk, K)
    if nDim == 3:
        assert np.array_equal(kd[:, 1], dirs[0])  # phi block first
        assert np.array_equal(kd[:, 0], dirs[1])  # then theta
    else:
        assert np.array_equal(kd[:, 0], dirs[0])
        assert (kd[:, 1] == 0).all()
    per_r = s[nblk * K:].reshape(Nmc, 2, K)  # per realization: gamma block, psi block
    assert np.array_equal(draws[:, :, 0], per_r[:, 0])
    assert np.array_equal(draws[:, :, 1], per_r[:, 1])
