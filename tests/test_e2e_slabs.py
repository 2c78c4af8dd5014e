"""The flat entry point into page-locked host memory copies the field out in
point slabs while the next slabs compute (rf_host.cu run_plan_slabs).  The
field must be bitwise the field of the plain path (pageable destination):
the same kernels on the same tiles, only launched per slab."""
import numpy as np
import pytest

import randomfield_b200 as rf
from tests.helpers import grid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,Nmc,kn", [("bf16", 8, (16, 16, 16)), ("fp16", 3, (12, 12, 12))])
def test_pinned_slabs_equal_the_plain_path(prec, Nmc, kn):
    torch = pytest.importorskip("torch")
    x = grid(72, 0.07)  # 373,248 points: 2,916 tiles, eight slabs on 148 SMs
    n = x.shape[0]
    kw = dict(precision=prec, k_nstep=kn, seed_start=4)
    plain = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "lognormal", (1.0, 0.8, 1.2), 1.0, 0.25,
                                                       Nmc, rf.SHINOZUKA, **kw)
    pinned_t = torch.empty((Nmc, n), dtype=torch.float64, pin_memory=True)
    pinned = pinned_t.numpy().T
    assert pinned.flags.f_contiguous
    rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "lognormal", (1.0, 0.8, 1.2), 1.0, 0.25, Nmc,
                                               rf.SHINOZUKA, randField=pinned, **kw)
    np.testing.assert_array_equal(pinned, plain)


def test_pinned_slabs_isotropic_table_path():
    torch = pytest.importorskip("torch")
    from tests.helpers import uniform_points

    x = uniform_points(380000, 9.0, seed=21)  # GEN_TABLE (isotropic), two slabs
    n, Nmc = x.shape[0], 5
    kw = dict(precision="bf16", iso_n_radial=32, iso_n_dir=32, seed_start=2)
    plain = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, Nmc,
                                                       rf.ISOTROPIC, **kw)
    pinned_t = torch.empty((Nmc, n), dtype=torch.float64, pin_memory=True)
    pinned = pinned_t.numpy().T
    rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, Nmc,
                                               rf.ISOTROPIC, randField=pinned, **kw)
    np.testing.assert_array_equal(pinned, plain)
