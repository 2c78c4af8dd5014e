"""rf_generate_device_noalloc, the allocation-free entry point.

It serves callers that must not allocate device memory while generating:
applications whose allocator (a caching pool, an OpenACC or CUDA Fortran
runtime) owns and has reserved nearly all device memory, or latency-critical
loops that cannot afford cudaMalloc's implicit synchronisation.  Its working
memory is one fixed 32 MiB device array per GPU shared by all calls.

Checked here through the C-ABI:
  - it runs the same table and contraction kernels on the same plan as the
    context entry point rf_generate_device, so two calls in a row give the
    context's field bit for bit (the normalised case only to 1e-12: its
    moments are FP64 sums whose atomic order varies from run to run);
  - the multi-block loop (more realizations than one launch holds), which
    reuses one scratch operand for every realization block;
  - a call right after one that left a larger operand and a wavevector table
    of another generator in the array, so that a stale read would show;
  - the field against the FP64 oracle within the suite's tolerances (plain
    FP32 max-abs <= 1e-5 * std, BF16 relative L2 <= 2e-3);
  - repeated calls take no device memory; a request larger than the scratch
    is rejected with RF_ESCRATCH.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.helpers import errors, grid, uniform_points

pytestmark = pytest.mark.gpu

CASES = [
    # (points, precision, Nmc, options)
    ("grid", "bf16", 4, dict(k_nstep=(16, 16, 16))),
    ("grid", "fp32", 4, dict(k_nstep=(16, 16, 16))),
    ("iso", "fp16", 16, dict(iso_n_radial=32, iso_n_dir=16)),
    # 160 realizations: two realization blocks of the BF16 hi/lo form (128 + 32)
    ("grid16", "bf16", 160, dict(k_nstep=(12, 12, 12))),
]


def _points(kind):
    if kind == "grid":
        return grid(24, 0.1)
    if kind == "grid16":
        return grid(16, 0.1)
    return uniform_points(20000, 8.0, seed=5)


def _device_run(fn, x, Nmc, method, prec, margi=1, avg=0.0, var=1.0, **opts):
    """The field [r, i] of one call of `fn` (the context or the no-allocation
    entry point) on device buffers."""
    import torch

    n, nDim = x.shape
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    out = torch.full((Nmc, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fn(dx, nDim, n, 1, margi, [1.0] * nDim, avg, var, Nmc, method, out, precision=prec, **opts)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _context_field(x, Nmc, method, prec, **kw):
    ctx = rf.Context(0)
    try:
        def fn(*a, **k):
            ctx.generate(*a, **k)
            ctx.synchronize()
        return _device_run(fn, x, Nmc, method, prec, **kw)
    finally:
        ctx.close()


def _noalloc_field(x, Nmc, method, prec, **kw):
    return _device_run(rf.generate_device_noalloc, x, Nmc, method, prec, **kw)


@pytest.mark.parametrize("kind,prec,Nmc,opts", CASES)
def test_noalloc_equals_context_entry_point(kind, prec, Nmc, opts):
    torch = pytest.importorskip("torch")
    x = _points(kind)
    n, nDim = x.shape
    method = rf.ISOTROPIC if kind == "iso" else rf.SHINOZUKA
    ref = _context_field(x, Nmc, method, prec, **opts)
    assert np.isfinite(ref).all()
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    for call in range(2):
        out = torch.full((Nmc, n), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rf.generate_device_noalloc(dx, nDim, n, 1, 1, [1.0] * nDim, 0.0, 1.0, Nmc, method, out, precision=prec,
                                   **opts)
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free0  # no device memory taken by the call
        got = out.cpu().numpy()
        assert np.array_equal(got, ref), (call, errors(got, ref))


def test_noalloc_after_a_larger_request_reads_no_stale_scratch():
    """A large GEN_GRID3 operand, then an isotropic (GEN_TABLE) request that
    also fills the wavevector table, then a small GEN_GRID3 request: each
    must equal the context entry point's field bit for bit."""
    big = grid(20, 0.1)
    small = grid(12, 0.1)
    iso = uniform_points(5000, 6.0, seed=9)
    _noalloc_field(big, 64, rf.SHINOZUKA, "bf16", k_nstep=(24, 24, 24))
    got_iso = _noalloc_field(iso, 8, rf.ISOTROPIC, "bf16", iso_n_radial=16, iso_n_dir=8)
    got_small = _noalloc_field(small, 4, rf.SHINOZUKA, "bf16", k_nstep=(8, 8, 8))
    ref_iso = _context_field(iso, 8, rf.ISOTROPIC, "bf16", iso_n_radial=16, iso_n_dir=8)
    ref_small = _context_field(small, 4, rf.SHINOZUKA, "bf16", k_nstep=(8, 8, 8))
    assert np.array_equal(got_iso, ref_iso), errors(got_iso, ref_iso)
    assert np.array_equal(got_small, ref_small), errors(got_small, ref_small)


def test_noalloc_normalised_lognormal_matches_context():
    """Normalisation uses the scratch's moment sums: two calls in a row agree
    with the context entry point to FP64 summation-order rounding."""
    x = grid(16, 0.1)
    kw = dict(margi=2, avg=1.0, var=0.25, k_nstep=(8, 8, 8), normalize=True)
    ref = _context_field(x, 12, rf.SHINOZUKA, "bf16", **kw)
    for _ in range(2):
        got = _noalloc_field(x, 12, rf.SHINOZUKA, "bf16", **kw)
        assert np.isfinite(got).all()
        assert errors(got, ref)[1] <= 1e-12, errors(got, ref)


@pytest.mark.parametrize("prec", ["bf16", "fp32"])
def test_noalloc_against_oracle(prec):
    x = grid(16, 0.1)
    ref = O.OracleRequest(x, Nmc=4, kNStep=(8, 8, 8)).generate()
    got = _noalloc_field(x, 4, rf.SHINOZUKA, prec, k_nstep=(8, 8, 8))
    if prec == "fp32":
        assert errors(got, ref)[0] <= 1e-5 * ref.std(), errors(got, ref)
    else:
        assert errors(got, ref)[1] <= 2e-3, errors(got, ref)


def test_noalloc_rejects_requests_beyond_scratch():
    torch = pytest.importorskip("torch")
    x = grid(8, 0.1)
    n, nDim = x.shape
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    out = torch.empty((256, n), dtype=torch.float64, device="cuda")
    with pytest.raises(rf.RandomFieldError) as e:
        # 32^3 x 4 wavevectors and 256 realizations: about 134 MB of tables
        rf.generate_device_noalloc(dx, nDim, n, 1, 1, [1.0] * 3, 0.0, 1.0, 256, rf.SHINOZUKA, out,
                                   precision="fp16", k_nstep=(32, 32, 32))
    assert e.value.code == -24 and "scratch" in str(e.value)
