"""Generates the small golden fixtures of tests/golden/ from the FP64 oracle.

    python tests/golden/make_golden.py

The reference (Fortran 90 + MPI + HDF5 + FFTW) ships no golden vectors and
cannot be compiled here, so these fixtures are oracle outputs: they freeze
the restated algorithm (rnglib stream, wavevector tables, draw order, sums,
marginal map) so that any change to the oracle or the GPU path shows up as a
diff.  Each case stores its inputs next to its output.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

CASES = {
    "shinozuka_grid": dict(pts=("grid", 8, 0.2, 3), kw=dict(Nmc=3, kNStep=(6, 5, 4))),
    "shinozuka_aniso_lognormal": dict(pts=("uniform", 400, 3.0, 3, 7),
                                      kw=dict(Nmc=2, kNStep=(5, 6, 4), corrL=(2.0, 1.0, 0.5),
                                              margiFirst=O.FOM_LOGNORMAL, fieldAvg=1.0, fieldVar=0.25)),
    "shinozuka_2d": dict(pts=("uniform", 300, 4.0, 2, 3), kw=dict(Nmc=3, kNStep=(7, 9), corrL=(0.7, 1.3))),
    "isotropic_3d": dict(pts=("uniform", 300, 4.0, 3, 4),
                         kw=dict(Nmc=3, method=O.ISOTROPIC, isoNRadial=12, isoNDir=7, seedStart=5)),
    "cm_cos": dict(pts=("grid", 6, 0.3, 3), kw=dict(Nmc=2, corrMod=O.CM_COS, kNStep=(8, 3, 3))),
    "literal": dict(pts=("grid", 6, 0.3, 3), kw=dict(Nmc=2, kNStep=(4, 4, 4), literal=True)),
    "normalized": dict(pts=("uniform", 500, 5.0, 3, 9), kw=dict(Nmc=2, kNStep=(5, 5, 5), normalize=True,
                                                                  fieldAvg=3.0, fieldVar=4.0)),
}


def points(spec):
    if spec[0] == "grid":
        _, n, h, nd = spec
        return O.grid([0.0] * nd, [h] * nd, [n] * nd)
    _, n, side, nd, seed = spec
    rs = np.random.RandomState(seed)
    return rs.uniform(0.0, side, size=(n, nd)).astype(np.float32).astype(np.float64)


def make(name):
    c = CASES[name]
    x = points(c["pts"])
    rq = O.OracleRequest(x, **c["kw"])
    return x, rq.generate()


def rng_stream():
    import ctypes as C

    out = {}
    for s in (0, 1, 99):
        r = O.rng(s)
        out[f"seed{s}"] = np.array([O.lib().rfo_rng_i4_uni(C.byref(r)) for _ in range(1000)], dtype=np.int64)
    return out


def main():
    for name in CASES:
        x, f = make(name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), xPoints=x, randField=f)
        print(name, x.shape, f.shape)
    np.savez_compressed(os.path.join(HERE, "rnglib_stream.npz"), **rng_stream())


if __name__ == "__main__":
    main()
