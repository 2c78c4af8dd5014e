"""Drives every entry point of the C oracle on small inputs; run by
tests/test_sanitizers.py in a child process with the AddressSanitizer/UBSan
build of the oracle (RFO_LIB) and libasan preloaded.  Prints "exercised"."""
import ctypes as C
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from oracle import oracle as O  # noqa: E402

L = O.lib()
# rnglib
r = O.rng(3)
[L.rfo_rng_i4_uni(C.byref(r)) for _ in range(100)]
[L.rfo_rng_r8_uni_01(C.byref(r)) for _ in range(100)]
L.rfo_rng_set_initial_seed(C.byref(r), 12345, 67890)
L.rfo_rng_init_generator(C.byref(r), 0)
L.rfo_rng_advance_state(C.byref(r), 10)
L.rfo_rng_cgn_set(C.byref(r), 2)
L.rfo_rng_i4_uni(C.byref(r))
O.rng(None)
assert L.rfo_multmod(40014, 12345, 2147483563) >= 0

# requests: Shinozuka 1-D to 3-D, isotropic, randomization, literal, cm_COS, lognormal + normalisation
x3 = O.grid([0.0, 0.0, 0.0], [0.1, 0.15, 0.2], [7, 6, 5])
x2 = O.grid([0.0, 0.0], [0.1, 0.2], [9, 8])
x1 = O.grid([0.5], [0.05], [40])
cases = [
    (x3, dict(Nmc=3, kNStep=(4, 3, 5))),
    (x3, dict(Nmc=2)),
    (x2, dict(Nmc=2, kNStep=(5, 4), margiFirst=O.FOM_LOGNORMAL, fieldAvg=1.0, fieldVar=0.25, normalize=True)),
    (x1, dict(Nmc=2)),
    (x3, dict(Nmc=2, method=O.ISOTROPIC, isoNRadial=6, isoNDir=5)),
    (x2, dict(Nmc=2, method=O.ISOTROPIC, isoNRadial=6, isoNDir=5)),
    (x3, dict(Nmc=2, method=3, kNStep=(4, 3, 3))),
    (x3, dict(Nmc=2, kNStep=(4, 3, 3), literal=True)),
    (x3, dict(Nmc=2, kNStep=(4, 3, 3), corrMod=O.CM_COS)),
]
for x, kw in cases:
    rq = O.OracleRequest(x, **kw)
    rq.geometry()
    rq.kpoints()
    rq.phase_matrix()
    f = rq.generate()
    rq.generate(rows=np.array([0, 3, x.shape[0] - 1]), nthreads=2)
    if not kw.get("literal"):  # the recast form refuses literal mode
        rq.generate(recast=True)
    assert np.isfinite(f).all()
rq = O.OracleRequest(x3, Nmc=2, kNStep=(4, 3, 3))
rq.baseline(0, 10, 0, 2, nthreads=2)
# marginal, normalisation, grid helpers
v = np.linspace(-2, 2, 50)
L.rfo_marginal(O.FOM_LOGNORMAL, 1.0, 0.25, v.ctypes.data_as(C.POINTER(C.c_double)), v.size)
w = np.random.RandomState(0).normal(size=(2, 30))
L.rfo_normalize(w.ctypes.data_as(C.POINTER(C.c_double)), 30, 2)
O.unity_partition([12, 10, 8], [3, 2, 2])
O.unity_partition([12, 10], [3, 2], faceMask=0x5)
L.rfo_overlap_npoints(0.65, 2.0, 0.05)
# the FFT method and statistics restatements (numpy over the oracle's rnglib)
O.fft_method_field((12, 10), (0.1, 0.2), (1.0, 1.0), seedStart=1)
f = O.OracleRequest(O.grid([0.0, 0.0, 0.0], [0.1, 0.1, 0.1], [8, 8, 8]), Nmc=2, kNStep=(4, 4, 4)).generate()
O.field_statistics(f.T.copy(order="F"), (8, 8, 8), (0.1, 0.1, 0.1))
print("exercised")
