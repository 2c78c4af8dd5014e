"""GPU parity: the CUDA path, called through the C-ABI, against the FP64
oracle on the same seeded inputs.

Tolerances (stated here and in the bench):
  plain FP32 form      max-abs <= 1e-5 * field std
  BF16 form           relative-L2 <= 2e-3 per realization (TF32 K-steps, or hi/lo B rows)
  FP16 form            relative-L2 <= 2e-3 per realization
  BF16 fast form       relative-L2 <= 3e-3 (single BF16 amplitude side)
  FP8 e4m3 form        relative-L2 <= 5e-2 (stated option: 3 significand bits in the trig tile)
Full-size workloads are checked on oracle row subsets plus size-independent
properties (moments of the whole field, determinism).
"""
import os

import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.golden import make_golden as G
from tests.helpers import errors, grid, per_realization_errors, uniform_points

pytestmark = pytest.mark.gpu

FP32_MAXABS = 1e-5
REL_L2 = {"bf16": 2e-3, "fp16": 2e-3, "bf16_fast": 3e-3, "fp8": 5e-2}
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gpu(x, prec, **kw):
    """Run the CUDA path; returns [r, i] like the oracle."""
    nDim = x.shape[1]
    corrL = kw.pop("corrL", (1.0,) * nDim)
    args = dict(corrMod=kw.pop("corrMod", 1), margiFirst=kw.pop("margiFirst", 1), fieldAvg=kw.pop("fieldAvg", 0.0),
                fieldVar=kw.pop("fieldVar", 1.0), Nmc=kw.pop("Nmc"), method=kw.pop("method", 2))
    out = rf.create_standard_gaussian_field_unstruct(x.T, args["corrMod"], args["margiFirst"], corrL,
                                                     args["fieldAvg"], args["fieldVar"], args["Nmc"], args["method"],
                                                     precision=prec, **kw)
    return np.asarray(out).T


def oracle(x, rows=None, **kw):
    okw = dict(kw)
    for a, b in (("k_nstep", "kNStep"), ("iso_n_radial", "isoNRadial"), ("iso_n_dir", "isoNDir"),
                 ("seed_start", "seedStart"), ("x_range", "xRange")):
        if a in okw:
            okw[b] = okw.pop(a)
    return O.OracleRequest(x, **okw).generate(rows=rows)


def check(prec, got, ref):
    """FP32: max-abs bound.  Tensor-core forms: the relative-L2 bound, over the
    whole compared field and for every realization on its own."""
    if prec == "fp32":
        mx, _ = errors(got, ref)
        assert mx <= FP32_MAXABS * ref.std(), (mx, ref.std())
    else:
        assert errors(got, ref)[1] <= REL_L2[prec]
        for r, (mx, rl2) in enumerate(per_realization_errors(got, ref)):
            assert rl2 <= REL_L2[prec], (r, rl2, mx)


# ------------------------------------------------------------------ configs
@pytest.fixture(scope="module")
def cfg1():
    x = grid(32, 0.1)
    kw = dict(Nmc=4, k_nstep=(16, 16, 16))
    rows = np.arange(0, x.shape[0], 7)
    return x, kw, rows, oracle(x, rows=rows, **kw)


@pytest.mark.parametrize("prec", ["fp32", "bf16", "fp16", "bf16_fast"])
def test_config1_shinozuka_32cubed(cfg1, prec):
    x, kw, rows, ref = cfg1
    got = gpu(x, prec, **kw)
    check(prec, got[:, rows], ref)


@pytest.fixture(scope="module")
def cfg2():
    x = uniform_points(200_000, 10.0, seed=2)
    kw = dict(Nmc=64, method=1, iso_n_radial=64, iso_n_dir=64, margiFirst=2, fieldAvg=1.0, fieldVar=0.25)
    rows = np.random.RandomState(0).choice(x.shape[0], 600, replace=False)
    return x, kw, rows, oracle(x, rows=rows, **kw)


@pytest.mark.parametrize("prec", ["fp32", "bf16", "fp16"])
def test_config2_isotropic_lognormal(cfg2, prec):
    x, kw, rows, ref = cfg2
    got = gpu(x, prec, **kw)[:, rows]
    if prec == "fp32":
        # lognormal: compare in the log domain (the Gaussian field before exp)
        mx, _ = errors(np.log(got), np.log(ref))
        assert mx <= FP32_MAXABS * np.log(ref).std(), mx
    else:
        for mx, rl2 in per_realization_errors(np.log(got), np.log(ref)):
            assert rl2 <= REL_L2[prec], rl2


@pytest.fixture(scope="module")
def cfg3():
    x = grid(128, 0.05)
    kw = dict(Nmc=64, k_nstep=(24, 24, 24), corrL=(2.0, 1.0, 0.5))
    rows = np.random.RandomState(1).choice(x.shape[0], 160, replace=False)
    return x, kw, rows, oracle(x, rows=rows, **kw)


@pytest.mark.parametrize("prec", ["bf16", "fp16", "fp32"])
def test_config3_shinozuka_128cubed(cfg3, prec):
    x, kw, rows, ref = cfg3
    got = gpu(x, prec, **kw)
    check(prec, got[:, rows], ref)
    if prec == "bf16":
        # size-independent: ensemble variance of the discrete sum
        rq = O.OracleRequest(x[:8], Nmc=1, kNStep=(24, 24, 24), corrL=(2.0, 1.0, 0.5),
                             xRange=tuple(x.max(0) - x.min(0)))
        g = rq.geometry()
        _, _, S = rq.kpoints()
        var_th = g.ampMult ** 2 / 2 * S.sum()
        assert got.var() == pytest.approx(var_th, rel=0.15)
        assert abs(got.mean()) < 0.15


# ---------------------------------------------------------------- fixtures
@pytest.mark.parametrize("name", sorted(G.CASES))
@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_golden_fixtures(name, prec):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = G.CASES[name]["kw"]
    kw = dict(Nmc=c["Nmc"], method=c.get("method", 2), corrMod=c.get("corrMod", 1),
              margiFirst=c.get("margiFirst", 1), fieldAvg=c.get("fieldAvg", 0.0), fieldVar=c.get("fieldVar", 1.0))
    x = z["xPoints"]
    if "corrL" in c:
        kw["corrL"] = c["corrL"]
    if "kNStep" in c:
        kw["k_nstep"] = tuple(c["kNStep"]) + (0,) * (3 - len(c["kNStep"]))
    for a, b in (("isoNRadial", "iso_n_radial"), ("isoNDir", "iso_n_dir"), ("seedStart", "seed_start"),
                 ("literal", "literal"), ("normalize", "normalize")):
        if a in c:
            kw[b] = c[a]
    got = gpu(x, prec, **kw)
    ref = z["randField"]
    if c.get("margiFirst", 1) == 2:
        got, ref = np.log(got), np.log(ref)
    if prec == "fp32":
        assert errors(got, ref)[0] <= FP32_MAXABS * max(ref.std(), 1e-300) * 10
    else:
        assert errors(got, ref)[1] <= REL_L2[prec]
        for r, (mx, rl2) in enumerate(per_realization_errors(got, ref)):
            assert rl2 <= REL_L2[prec], (name, r, rl2)


# -------------------------------------------------------------- edge cases
def test_cm_cos_known_answer_on_gpu():
    x = grid(6, 0.3)
    rq = O.OracleRequest(x, corrMod=O.CM_COS, Nmc=3, kNStep=(8, 3, 3))
    g = rq.geometry()
    z = np.load(os.path.join(GOLDEN, "rnglib_stream.npz"))["seed0"]
    for prec in ("fp32", "bf16", "fp16"):
        got = gpu(x, prec, Nmc=3, corrMod=2, k_nstep=(8, 3, 3))
        for r in range(3):
            phi = 2.0 * 3.1415926535898 * (z[r * g.K + 5] * 4.656613057e-10)
            want = g.ampMult * np.cos(x[:, 0] * 5 * g.kDelta[0] + phi)
            if prec == "fp32":
                np.testing.assert_allclose(got[r], want, atol=1e-6 * g.ampMult)
            else:  # the stated bound of the 16-bit forms, per realization
                assert errors(got[r], want)[1] <= REL_L2[prec], (prec, r, errors(got[r], want))


@pytest.mark.parametrize("n,Nmc", [(1000, 1), (129, 17), (4097, 33), (77, 130)])
def test_ragged_sizes(n, Nmc):
    x = uniform_points(n, 3.0, seed=n)
    kw = dict(Nmc=Nmc, k_nstep=(5, 6, 7))
    ref = oracle(x, **kw)
    for prec in ("fp32", "bf16"):
        check(prec, gpu(x, prec, **kw), ref)


def test_single_point_with_explicit_extent():
    x = np.array([[0.3, 0.1, 0.7]])
    kw = dict(Nmc=5, k_nstep=(4, 4, 4), x_range=(2.0, 2.0, 2.0))
    ref = oracle(x, **kw)
    check("fp32", gpu(x, "fp32", **kw), ref)


def test_zero_extent_rejected_on_gpu():
    x = np.zeros((10, 3))
    with pytest.raises(rf.RandomFieldError) as e:
        gpu(x, "bf16", Nmc=2)
    assert e.value.code == -8


@pytest.mark.parametrize("nDim,method", [(1, 2), (2, 2), (2, 1), (3, 1)])
def test_table_generator_dimensions(nDim, method):
    x = uniform_points(3000, 5.0, nDim=nDim, seed=nDim + 10 * method)
    kw = dict(Nmc=8, method=method, corrL=(1.0, 0.8, 1.2)[:nDim])
    if method == 2:
        kw["k_nstep"] = (40, 9, 0)[:nDim] + (0,) * (3 - nDim)
    else:
        kw.update(iso_n_radial=20, iso_n_dir=16)
    ref = oracle(x, **kw)
    for prec in ("fp32", "bf16", "fp16"):
        check(prec, gpu(x, prec, **kw), ref)


def test_grid3_large_axis_falls_back_to_table():
    x = uniform_points(2000, 8.0, seed=3)
    kw = dict(Nmc=4, k_nstep=(40, 5, 6))
    ref = oracle(x, **kw)
    check("bf16", gpu(x, "bf16", **kw), ref)


def test_literal_mode_two_slabs():
    # K = 32^3 * 4 -> xSlab = int(3e8 / K) = 2288 rows: 2 slabs for 4000 points
    x = uniform_points(4000, 6.0, seed=8)
    kw = dict(Nmc=2, k_nstep=(32, 32, 32), literal=True)
    rows = np.array([0, 5, 2287, 2288, 2300, 3999])
    ref = oracle(x, rows=rows, **kw)
    got = gpu(x, "fp32", **kw)[:, rows]
    assert errors(got, ref)[0] <= 1e-5 * max(1.0, np.abs(ref).max())


def test_normalize_and_lognormal():
    x = uniform_points(5000, 6.0, seed=4)
    kw = dict(Nmc=3, k_nstep=(6, 6, 6), normalize=True, margiFirst=2, fieldAvg=2.0, fieldVar=0.5)
    ref = oracle(x, **kw)
    got = gpu(x, "fp32", **kw)
    np.testing.assert_allclose(np.log(got), np.log(ref), atol=1e-5)


def test_seed_start_and_determinism():
    x = uniform_points(3000, 4.0, seed=6)
    kw = dict(Nmc=4, k_nstep=(8, 8, 8), seed_start=42)
    a = gpu(x, "bf16", **kw)
    b = gpu(x, "bf16", **kw)
    np.testing.assert_array_equal(a, b)
    check("bf16", a, oracle(x, **kw))
    c = gpu(x, "bf16", Nmc=4, k_nstep=(8, 8, 8), seed_start=43)
    assert not np.allclose(a, c)


def test_device_api_matches_flat_api():
    torch = pytest.importorskip("torch")
    x = grid(20, 0.1)
    kw = dict(k_nstep=(12, 12, 12))
    flat = rf.create_standard_gaussian_field_unstruct(x.T, 1, 1, [1, 1, 1], 0.0, 1.0, 8, 2, precision="bf16", **kw)
    ctx = rf.Context(0)
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dout = torch.empty((8, x.shape[0]), dtype=torch.float64, device="cuda")  # column-major n x Nmc
    ctx.generate(dx, 3, x.shape[0], 1, 1, [1, 1, 1], 0.0, 1.0, 8, 2, dout, precision="bf16", **kw)
    ctx.synchronize()
    np.testing.assert_array_equal(dout.cpu().numpy(), np.asarray(flat).T)
    ctx.close()


# --------------------------------------------------- randomization (method 3)
@pytest.mark.parametrize("prec", ["fp32", "bf16"])
@pytest.mark.parametrize("nDim", [2, 3])
def test_randomization_method(prec, nDim):
    """Method 3: uniformly random wavevectors (drawn before the phases), the
    Shinozuka sum over them, through GEN_TABLE."""
    x = uniform_points(4000, 5.0, nDim=nDim, seed=31)
    kw = dict(Nmc=6, method=3, k_nstep=(10, 10, 10)[:nDim] + (0,) * (3 - nDim), seed_start=4)
    rows = np.random.RandomState(2).choice(x.shape[0], 200, replace=False)
    ref = oracle(x, rows=rows, **kw)
    got = gpu(x, prec, **kw)
    check(prec, got[:, rows], ref)


def test_randomization_literal_mode():
    x = uniform_points(3000, 4.0, seed=8)
    kw = dict(Nmc=3, method=3, k_nstep=(8, 8, 8), seed_start=2, literal=True)
    ref = oracle(x, **kw)
    got = gpu(x, "fp32", **kw)
    check("fp32", got, ref)


# ---------------------------------------------------------- FP8 e4m3 option
@pytest.mark.parametrize("kind", ["grid3", "table", "isotropic"])
def test_fp8_form(kind):
    """kind::f8f6f4 MMAs on e4m3 trig tiles and hi/lo e4m3 amplitude rows:
    GEN_GRID3 (24 wavenumbers on axis 3), GEN_TABLE (Shinozuka 2-D) and the
    isotropic table, against the oracle within the option's stated bound."""
    if kind == "grid3":
        x = grid(24, 0.1)
        kw = dict(Nmc=64, k_nstep=(24, 24, 24), seed_start=2)
    elif kind == "table":
        x = uniform_points(5000, 4.0, nDim=2, seed=5)
        kw = dict(Nmc=20, k_nstep=(32, 32, 0), seed_start=3)
    else:
        x = uniform_points(8000, 8.0, seed=6)
        kw = dict(Nmc=33, method=1, iso_n_radial=40, iso_n_dir=40, seed_start=4)
    rows = np.random.RandomState(3).choice(x.shape[0], 160, replace=False)
    ref = oracle(x, rows=rows, **kw)
    got = gpu(x, "fp8", **kw)
    check("fp8", got[:, rows], ref)
    # the form is an option: its error is well above the BF16 form's
    assert errors(got[:, rows], ref)[1] > 2e-3
