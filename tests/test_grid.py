"""The structured-grid path (rf_generate_grid): the Shinozuka sum evaluated
axis by axis on a tensor grid of points.

CPU: the axis-by-axis factorisation restated in numpy from the oracle's own
wavevectors and phases (C_k = Bc_k - i Bs_k, k = q kn + i1 + n1 (i2 + n2 i3))
equals the oracle's point-by-point sum on small grids in 1-D, 2-D and 3-D.
GPU: the device field equals the FP64 oracle on the grid's points to FP64
rounding (relative-L2 <= 1e-11 per realization) across dimensions, extents
that span several row and column blocks, both marginals, cm_COS, the
reference's wavenumber rule and explicit counts, normalisation and seeds;
the point path on the same points agrees within its own form's tolerance;
unsupported requests are refused with RF_ENOTSUP, invalid ones with their
codes.
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O

GRID_REL_L2 = 1e-11


def _oracle(xMin, xStep, xNStep, corrL, **kw):
    x = O.grid(xMin, xStep, xNStep)
    req = O.OracleRequest(x, corrL=corrL, **kw)
    return req, req.generate()


def _separable_numpy(req, xMin, xStep, xNStep):
    """Axis-by-axis evaluation from the oracle's wavevector grid and phases."""
    g = req.geometry()
    nd = req.nDim
    R = req.req.Nmc
    Bc, Bs = req.phase_matrix()
    C = Bc - 1j * Bs  # a_k exp(i phi_k)
    kn = [g.kNStep[d] if d < nd else 1 for d in range(3)]
    S2 = 2 if nd >= 2 else 1
    S3 = 2 if nd == 3 else 1
    C = C.reshape(R, S2, S3, kn[2], kn[1], kn[0])  # q = s2 S3 + s3, then i3, i2, i1
    E = []
    for d in range(3):
        if d < nd:
            j = np.arange(xNStep[d])
            xd = (xMin[d] + xStep[d] * j) / req.req.corrL[d]
            kd = g.kDelta[d] * np.arange(kn[d])
            E.append(np.exp(1j * np.outer(kd, xd)))  # [i, j]
        else:
            E.append(np.ones((1, 1), dtype=complex))
    N = [xNStep[d] if d < nd else 1 for d in range(3)]
    # axis 3: both signs of k3
    G = np.einsum("rakji,kz->razji", C[:, :, 0], E[2])
    if S3 == 2:
        G = G + np.einsum("rakji,kz->razji", C[:, :, 1], np.conj(E[2]))
    # axis 2
    H = np.einsum("rzji,jy->rzyi", G[:, 0], E[1])
    if S2 == 2:
        H = H + np.einsum("rzji,jy->rzyi", G[:, 1], np.conj(E[1]))
    f = g.ampMult * np.real(np.einsum("rzyi,ix->rzyx", H, E[0]))
    return f.reshape(R, N[0] * N[1] * N[2])


@pytest.mark.parametrize("xNStep,kn", [((9,), (7,)), ((8, 6), (5, 4)), ((7, 6, 5), (4, 3, 5))])
def test_separable_restatement_matches_oracle(xNStep, kn):
    nd = len(xNStep)
    xMin = [0.3, -1.0, 2.0][:nd]
    xStep = [0.21, 0.17, 0.3][:nd]
    corrL = [1.0, 2.0, 0.5][:nd]
    req, ref = _oracle(xMin, xStep, xNStep, corrL, Nmc=2, kNStep=kn, seedStart=4)
    f = _separable_numpy(req, xMin, xStep, xNStep)
    np.testing.assert_allclose(f, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def ctx():
    c = rf.Context(0)
    yield c
    c.close()


def _device(ctx, xMin, xStep, xNStep, corrL, Nmc, corrMod=1, margiFirst=1, fieldAvg=0.0, fieldVar=1.0, **kw):
    torch = pytest.importorskip("torch")
    n = int(np.prod(xNStep))
    d = torch.full((Nmc, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the fill runs on torch's stream, the field on the context's
    ctx.generate_grid(d, xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, **kw)
    torch.cuda.synchronize()
    return d.cpu().numpy()


CASES = [
    # xMin, xStep, xNStep, corrL, Nmc, kNStep (0: the reference rule), extra
    ((0.3, -1.0, 2.0), (0.1, 0.15, 0.2), (20, 17, 13), (1.0, 2.0, 0.5), 3, (6, 5, 7), {}),
    ((0.0, 0.0, 0.0), (0.05, 0.05, 0.05), (24, 20, 16), (0.5, 0.5, 0.5), 2, (0, 0, 0), {}),
    ((0.0, 0.0, 0.0), (0.02, 0.1, 0.1), (300, 3, 2), (1.0, 1.0, 1.0), 2, (9, 4, 3), {}),
    ((0.0, 0.0, 0.0), (0.1, 0.01, 0.1), (5, 150, 2), (1.0, 1.0, 1.0), 2, (3, 8, 3), {}),
    ((0.0, 0.0, 0.0), (0.1, 0.1, 0.01), (3, 2, 130), (1.0, 1.0, 1.0), 2, (3, 3, 10), {}),
    ((-2.0, 1.0), (0.07, 0.11), (70, 45), (1.0, 2.0), 4, (12, 9), dict(margiFirst=2, fieldAvg=1.0, fieldVar=0.25)),
    ((0.5,), (0.01,), (300,), (0.8,), 3, (0,), {}),
    ((0.0, 0.0, 0.0), (0.2, 0.2, 0.2), (11, 9, 8), (1.0, 1.0, 1.0), 2, (4, 4, 4), dict(corrMod=2)),
    ((0.0, 0.0, 0.0), (0.1, 0.1, 0.1), (16, 12, 10), (1.0, 1.0, 1.0), 3, (5, 5, 5), dict(normalize=True)),
    ((0.0, 0.0, 0.0), (0.1, 0.1, 0.1), (10, 9, 7), (1.0, 1.0, 1.0), 70, (4, 3, 3), dict(seed_start=7)),
    ((0.0, 0.0, 0.0), (0.05, 0.05, 0.05), (17, 13, 9), (2.0, 1.0, 0.5), 2, (24, 24, 24), {}),
    ((0.1, 0.2, 0.3), (0.3, 0.2, 0.1), (9, 8, 7), (1.0, 1.0, 1.0), 1, (32, 32, 32), {}),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_grid_matches_oracle(ctx, case):
    xMin, xStep, xNStep, corrL, Nmc, kn, extra = CASES[case]
    extra = dict(extra)
    corrMod = extra.pop("corrMod", 1)
    margiFirst = extra.pop("margiFirst", 1)
    fieldAvg = extra.pop("fieldAvg", 0.0)
    fieldVar = extra.pop("fieldVar", 1.0)
    normalize = extra.pop("normalize", False)
    seed = extra.pop("seed_start", 0)
    _, ref = _oracle(xMin, xStep, xNStep, corrL, Nmc=Nmc, kNStep=kn, seedStart=seed, corrMod=corrMod,
                     margiFirst=margiFirst, fieldAvg=fieldAvg, fieldVar=fieldVar, normalize=normalize)
    got = _device(ctx, xMin, xStep, xNStep, corrL, Nmc, corrMod=corrMod, margiFirst=margiFirst, fieldAvg=fieldAvg,
                  fieldVar=fieldVar, k_nstep=kn, seed_start=seed, normalize=normalize)
    assert np.isfinite(got).all()
    for r in range(Nmc):
        err = np.linalg.norm(got[r] - ref[r]) / np.linalg.norm(ref[r])
        assert err <= GRID_REL_L2, (r, err)


@pytest.mark.gpu
def test_grid_agrees_with_point_path(ctx):
    """The same field through rf_generate_device on the grid's points."""
    torch = pytest.importorskip("torch")
    xMin, xStep, xNStep, corrL = (0.0, 0.0, 0.0), (0.1, 0.1, 0.1), (32, 32, 32), (1.0, 1.0, 1.0)
    Nmc, kn = 4, (16, 16, 16)
    x = torch.from_numpy(O.grid(xMin, xStep, xNStep)).cuda()
    n = x.shape[0]
    g = _device(ctx, xMin, xStep, xNStep, corrL, Nmc, k_nstep=kn)
    for prec, tol in (("fp32", 1e-5), ("bf16", 2e-3)):
        d = torch.empty((Nmc, n), dtype=torch.float64, device="cuda")
        ctx.generate(x, 3, n, 1, 1, corrL, 0.0, 1.0, Nmc, 2, d, precision=prec, k_nstep=kn)
        torch.cuda.synchronize()
        p = d.cpu().numpy()
        for r in range(Nmc):
            assert np.linalg.norm(p[r] - g[r]) / np.linalg.norm(g[r]) <= tol, (prec, r)
    # the oracle on a row subset of this 32^3 x 16^3 x 4 workload
    rows = np.random.RandomState(3).choice(n, 256, replace=False)
    req = O.OracleRequest(O.grid(xMin, xStep, xNStep), corrL=corrL, Nmc=Nmc, kNStep=kn)
    ref = req.generate(rows=rows)
    assert np.abs(g[:, rows] - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.gpu
def test_grid_deterministic_and_stream(ctx):
    torch = pytest.importorskip("torch")
    args = ((0.0, 0.0, 0.0), (0.1, 0.1, 0.1), (40, 30, 20), (1.0, 1.0, 1.0), 5)
    a = _device(ctx, *args, k_nstep=(8, 8, 8))
    s = torch.cuda.Stream()
    d = torch.empty((5, 40 * 30 * 20), dtype=torch.float64, device="cuda")
    with torch.cuda.stream(s):
        ctx.generate_grid(d, *args[:3], 1, 1, (1.0, 1.0, 1.0), 0.0, 1.0, 5, k_nstep=(8, 8, 8), stream=s)
    s.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), a)


@pytest.mark.gpu
def test_grid_refusals(ctx):
    torch = pytest.importorskip("torch")
    d = torch.empty((1, 1000), dtype=torch.float64, device="cuda")
    base = ((0.0, 0.0, 0.0), (0.1, 0.1, 0.1), (10, 10, 10))

    def call(**kw):
        a = dict(xMin=base[0], xStep=base[1], xNStep=base[2], corrMod=1, margiFirst=1, corrL=(1.0, 1.0, 1.0),
                 fieldAvg=0.0, fieldVar=1.0, Nmc=1)
        opts = {k: kw.pop(k) for k in list(kw) if k in ("k_nstep", "literal", "normalize")}
        a.update(kw)
        ctx.generate_grid(d, **a, **opts)

    for kw, code in ((dict(method=1), -10), (dict(method=3), -10), (dict(literal=True), -10),
                     (dict(k_nstep=(40, 4, 4)), -10), (dict(Nmc=0), -1), (dict(corrL=(1.0, 0.0, 1.0)), -3),
                     (dict(xStep=(0.1, -0.1, 0.1)), -9), (dict(margiFirst=2, fieldAvg=0.0), -4),
                     (dict(method=7), -5)):
        with pytest.raises(rf.RandomFieldError) as e:
            call(**kw)
        assert e.value.code == code, kw


@pytest.mark.gpu
def test_grid_host_entry_point(ctx):
    """rf_create_standard_gaussian_field_grid (host randField) equals the
    device entry point, and refuses what the device entry point refuses."""
    xMin, xStep, xNStep, corrL = (0.0, 0.5, -1.0), (0.1, 0.2, 0.05), (30, 20, 40), (1.0, 2.0, 0.5)
    dev = _device(ctx, xMin, xStep, xNStep, corrL, 6, margiFirst=2, fieldAvg=1.0, fieldVar=0.25,
                  k_nstep=(10, 9, 12), seed_start=3)
    host = rf.create_standard_gaussian_field_grid(xMin, xStep, xNStep, 1, 2, corrL, 1.0, 0.25, 6,
                                                  k_nstep=(10, 9, 12), seed_start=3)
    assert host.shape == (30 * 20 * 40, 6) and host.flags.f_contiguous
    np.testing.assert_array_equal(host.T, dev)
    out = np.zeros((30 * 20 * 40, 6), order="F")
    rf.create_standard_gaussian_field_grid(xMin, xStep, xNStep, 1, 2, corrL, 1.0, 0.25, 6, randField=out,
                                           k_nstep=(10, 9, 12), seed_start=3)
    np.testing.assert_array_equal(out, host)
    with pytest.raises(rf.RandomFieldError) as e:
        rf.create_standard_gaussian_field_grid(xMin, xStep, xNStep, 1, 1, corrL, 0.0, 1.0, 2, method=1)
    assert e.value.code == -10
