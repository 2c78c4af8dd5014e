"""Shared workloads and error metrics of the test suite."""
import numpy as np

from oracle import oracle as O


def grid(n_per_axis, spacing, nDim=3, origin=0.0):
    """setGrid coordinates (axis 1 fastest) as n x nDim."""
    return O.grid([origin] * nDim, [spacing] * nDim, [n_per_axis] * nDim)


def uniform_points(n, side, nDim=3, seed=1234):
    rs = np.random.RandomState(seed)
    return rs.uniform(0.0, side, size=(n, nDim)).astype(np.float32).astype(np.float64)


def errors(gpu, ref):
    """(max-abs, relative-L2) of gpu vs ref, arrays [r, i]."""
    d = np.asarray(gpu, dtype=np.float64) - np.asarray(ref, dtype=np.float64)
    return float(np.abs(d).max()), float(np.linalg.norm(d) / np.linalg.norm(ref))


def per_realization_errors(gpu, ref):
    out = []
    for r in range(ref.shape[0]):
        out.append(errors(gpu[r], ref[r]))
    return out


def separable_field(xMin, xStep, xNStep, corrL, Nmc, kNStep=(0, 0, 0), seedStart=0, corrMod=O.CM_GAUSSIAN):
    """The Shinozuka field on the structured grid xMin + j xStep (axis 1
    fastest) from the oracle's own wavevectors and phases, evaluated axis by
    axis with complex matrix products (FP64): the whole field of a large grid
    in seconds, for full-field comparisons.  Returns [r, i] before the
    marginal map.  Pinned against the oracle's point-by-point sum in
    tests/test_full_field.py."""
    nd = len(xNStep)
    xr = tuple((xNStep[d] - 1) * xStep[d] for d in range(nd))
    req = O.OracleRequest(np.asarray(xMin, dtype=np.float64).reshape(1, nd), corrL=corrL, Nmc=Nmc, kNStep=kNStep,
                          seedStart=seedStart, corrMod=corrMod, xRange=xr)
    g = req.geometry()
    Bc, Bs = req.phase_matrix()  # [r, k]: a cos(phi), -a sin(phi)
    R = Nmc
    kn = [g.kNStep[d] if d < nd else 1 for d in range(3)]
    S2 = 2 if nd >= 2 else 1
    S3 = 2 if nd == 3 else 1
    N = [xNStep[d] if d < nd else 1 for d in range(3)]
    C = (Bc - 1j * Bs).reshape(R, S2, S3, kn[2], kn[1] * kn[0])  # k = q kn + i1 + n1 (i2 + n2 i3), q = s2 S3 + s3
    E = []
    for d in range(3):
        if d < nd:
            xd = (xMin[d] + xStep[d] * np.arange(N[d])) / corrL[d]
            E.append(np.exp(1j * np.outer(g.kDelta[d] * np.arange(kn[d]), xd)))  # [i, j]
        else:
            E.append(np.ones((1, 1), dtype=complex))
    G = np.matmul(E[2].T, C[:, :, 0])  # (R, S2, N3, k2 k1)
    if S3 == 2:
        G = G + np.matmul(np.conj(E[2]).T, C[:, :, 1])
    G = G.reshape(R, S2, N[2], kn[1], kn[0]).transpose(0, 1, 2, 4, 3)  # (R, S2, N3, k1, k2)
    H = np.matmul(G[:, 0], E[1])  # (R, N3, k1, N2)
    if S2 == 2:
        H = H + np.matmul(G[:, 1], np.conj(E[1]))
    H = H.transpose(0, 1, 3, 2)  # (R, N3, N2, k1)
    f = np.matmul(H.real, E[0].real) - np.matmul(H.imag, E[0].imag)  # (R, N3, N2, N1)
    return g.ampMult * f.reshape(R, -1)
