"""Localization blend on the GPU against the FP64 oracle.

The oracle assembles the group field the reference's way: every subdomain
field (seed seedStart + fieldNumber, its own grid and xRange) times the
subdomain partition of unity with all faces ramped (rfo_unity_partition,
localization_RF.f90:705-857), added into the group at its offset
(add_RF_to_Group, :199-263), then divided by the group partition of the
border faces (calls_RF.f90:324-369) and mapped to the marginal.  The GPU
field must match within the BF16 bound (relative-L2 <= 2e-3 on the Gaussian
field).  Shinozuka blends run through the structured-grid path (each
subdomain summed axis by axis in FP64), which must match to FP64 rounding;
the grouped-launch path (isotropic) within the BF16 bound.
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.helpers import errors

pytestmark = pytest.mark.gpu


def oracle_blend(G, h, F, Ov, L, Nmc, seed, corrL, kn, method=2, iso=(0, 0)):
    nd = len(G)
    group = np.zeros((Nmc, int(np.prod(G))))
    up_sub = O.unity_partition(L, Ov)
    nf = int(np.prod(F))
    for f in range(nf):
        fi = [f % F[0], (f // F[0]) % F[1] if nd > 1 else 0, f // (F[0] * F[1]) if nd > 2 else 0][:nd]
        org = [fi[d] * (L[d] - max(Ov[d], 0)) for d in range(nd)]
        pts = O.grid([org[d] * h[d] for d in range(nd)], h, L)
        rq = O.OracleRequest(pts, Nmc=Nmc, corrL=corrL, seedStart=seed + f + 1, kNStep=kn, method=method,
                             isoNRadial=iso[0], isoNDir=iso[1],
                             xRange=tuple((L[d] - 1) * h[d] for d in range(nd)) + (0.0,) * (3 - nd))
        sub = rq.generate() * up_sub[None, :]
        idx = np.arange(int(np.prod(L)))
        i = [idx % L[0], (idx // L[0]) % L[1], idx // (L[0] * L[1])][:nd]
        gi = (org[0] + i[0])
        if nd > 1:
            gi = gi + G[0] * (org[1] + i[1])
        if nd > 2:
            gi = gi + G[0] * G[1] * (org[2] + i[2])
        group[:, gi] += sub
    return group / O.unity_partition(G, Ov)[None, :]


@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_blend_3d_matches_oracle(prec):
    G, h, F, overlap = (21, 21, 21), (0.1, 0.1, 0.1), (2, 2, 2), 0.4
    grid = rf.BlendGrid.make(G, h, F, overlap)
    L, Ov = rf.blend_layout(grid, (1.0, 1.0, 1.0))
    assert (L, Ov) == ([12, 12, 12], [3, 3, 3])
    Nmc, seed, kn = 2, 5, (12, 12, 12)
    ctx = rf.Context(0)
    got = ctx.generate_blended(grid, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, Nmc, 2, precision=prec,
                               seed_start=seed, k_nstep=kn)
    ref = oracle_blend(G, h, F, Ov, L, Nmc, seed, (1.0, 1.0, 1.0), kn)
    assert np.isfinite(got).all()
    assert errors(got.T, ref)[1] <= 1e-11  # the structured-grid path: FP64 throughout
    # lognormal marginal after the border correction, on the device entry point
    torch = pytest.importorskip("torch")
    dout = torch.empty((Nmc, int(np.prod(G))), dtype=torch.float64, device="cuda")
    ctx.generate_blended_device(grid, "gaussian", "lognormal", (1.0, 1.0, 1.0), 1.0, 0.25, Nmc, 2, dout,
                                precision=prec, seed_start=seed, k_nstep=kn)
    ctx.synchronize()
    nv = np.log(1 + 0.25)
    lg = dout.cpu().numpy()
    assert errors((np.log(lg) - (0.0 - nv / 2)) / np.sqrt(nv), ref)[1] <= 1e-10
    ctx.close()


def test_blend_2d_isotropic_matches_oracle():
    G, h, F, overlap = (34, 26), (0.1, 0.1), (3, 2), 0.5
    grid = rf.BlendGrid.make(G, h, F, overlap)
    L, Ov = rf.blend_layout(grid, (1.0, 1.0))
    Nmc, seed = 3, 9
    ctx = rf.Context(0)
    got = ctx.generate_blended(grid, "gaussian", "gaussian", (1.0, 1.0), 0.0, 1.0, Nmc, 1, precision="bf16",
                               seed_start=seed, iso_n_radial=24, iso_n_dir=24)
    ref = oracle_blend(G, h, F, Ov, L[:2], Nmc, seed, (1.0, 1.0), (0, 0, 0), method=1, iso=(24, 24))
    assert errors(got.T, ref)[1] <= 2e-3
    ctx.close()


def test_single_field_blend_is_the_plain_field():
    """nFields = 1 everywhere: no ramps, the blend is the plain generation
    on the grid with seed seedStart + 1."""
    G, h = (16, 16, 16), (0.1, 0.1, 0.1)
    grid = rf.BlendGrid.make(G, h, (1, 1, 1), 0.0)
    ctx = rf.Context(0)
    got = ctx.generate_blended(grid, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, 4, 2, precision="bf16",
                               seed_start=3, k_nstep=(16, 16, 16))
    pts = O.grid([0.0] * 3, h, G)
    plain = rf.create_standard_gaussian_field_unstruct(pts.T, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, 4,
                                                       2, precision="bf16", seed_start=4, k_nstep=(16, 16, 16))
    assert errors(got, np.asarray(plain))[1] <= 2e-3
    ctx.close()
