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
    """The oracle's whole-grid FP64 reference (oracle.separable_field)."""
    return O.separable_field(xMin, xStep, xNStep, corrL, Nmc, kNStep=kNStep, seedStart=seedStart, corrMod=corrMod)
