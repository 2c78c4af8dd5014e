"""ctypes front end of the FP64 CPU oracle (oracle/rf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by the CPU baseline leg of ``bench.py``.  The product in
``randomfield_b200/`` never imports it.

Parity status: unpinned against reference output (the Fortran reference ships
no golden vectors and cannot be compiled here); see rf_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librfo.so")
# RFO_LIB names another build of the same library (the sanitizer build of
# `make -C oracle sanitize`); it is loaded as it is, never rebuilt here.
_LIB_OVERRIDE = os.environ.get("RFO_LIB")

ISOTROPIC, SHINOZUKA, RANDOMIZATION = 1, 2, 3
CM_GAUSSIAN, CM_COS = 1, 2
FOM_GAUSSIAN, FOM_LOGNORMAL = 1, 2


class Request(C.Structure):
    _fields_ = [
        ("nDim", C.c_int32),
        ("n", C.c_int64),
        ("xPoints", C.POINTER(C.c_double)),
        ("corrMod", C.c_int32),
        ("margiFirst", C.c_int32),
        ("corrL", C.c_double * 3),
        ("fieldAvg", C.c_double),
        ("fieldVar", C.c_double),
        ("Nmc", C.c_int32),
        ("method", C.c_int32),
        ("seedStart", C.c_int64),
        ("kNStep", C.c_int32 * 3),
        ("isoNRadial", C.c_int32),
        ("isoNDir", C.c_int32),
        ("literal", C.c_int32),
        ("normalize", C.c_int32),
        ("xRange", C.c_double * 3),
    ]


class Geometry(C.Structure):
    _fields_ = [
        ("nDim", C.c_int32),
        ("K", C.c_int64),
        ("kNStep", C.c_int32 * 3),
        ("kDelta", C.c_double * 3),
        ("kMax", C.c_double),
        ("ampMult", C.c_double),
        ("xRangeNorm", C.c_double * 3),
        ("xSlab", C.c_int64),
    ]


class RNG(C.Structure):
    _fields_ = [(nm, C.c_int32 * 32) for nm in ("ig1", "ig2", "lg1", "lg2", "cg1", "cg2", "anti")] + [
        ("g", C.c_int32),
        ("initialized", C.c_int32),
    ]


_lib = None


def build() -> None:
    """Compile librfo.so with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if _LIB_OVERRIDE:
            L = C.CDLL(_LIB_OVERRIDE)
        else:
            if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(HERE, "rf_oracle.c")
            ):
                build()
            L = C.CDLL(LIB_PATH)
        P = C.POINTER
        d = C.c_double
        L.rfo_multmod.argtypes = [C.c_int32] * 3
        L.rfo_multmod.restype = C.c_int32
        L.rfo_rng_seed.argtypes = [P(RNG), C.c_int64]
        L.rfo_rng_initialize.argtypes = [P(RNG)]
        L.rfo_rng_set_initial_seed.argtypes = [P(RNG), C.c_int32, C.c_int32]
        L.rfo_rng_init_generator.argtypes = [P(RNG), C.c_int32]
        L.rfo_rng_advance_state.argtypes = [P(RNG), C.c_int32]
        L.rfo_rng_cgn_set.argtypes = [P(RNG), C.c_int32]
        L.rfo_rng_i4_uni.argtypes = [P(RNG)]
        L.rfo_rng_i4_uni.restype = C.c_int32
        L.rfo_rng_i4_stream.argtypes = [P(RNG), C.c_int64, P(C.c_int32)]
        L.rfo_rng_i4_stream.restype = None
        L.rfo_rng_r8_uni_01.argtypes = [P(RNG)]
        L.rfo_rng_r8_uni_01.restype = d
        L.rfo_geometry_of.argtypes = [P(Request), P(Geometry)]
        L.rfo_kpoints.argtypes = [P(Request), P(d), P(d), P(d)]
        L.rfo_phase_matrix.argtypes = [P(Request), P(d), P(d)]
        L.rfo_generate.argtypes = [P(Request), P(C.c_int64), C.c_int64, P(d), C.c_int32]
        L.rfo_generate_recast.argtypes = [P(Request), P(C.c_int64), C.c_int64, P(d), C.c_int32]
        L.rfo_marginal.argtypes = [C.c_int32, d, d, P(d), C.c_int64]
        L.rfo_normalize.argtypes = [P(d), C.c_int64, C.c_int32]
        L.rfo_set_grid.argtypes = [C.c_int32, P(d), P(d), P(C.c_int32), P(d)]
        L.rfo_unity_partition.argtypes = [C.c_int32, P(C.c_int32), P(C.c_int32), C.c_uint32, P(d)]
        L.rfo_overlap_npoints.argtypes = [d, d, d]
        L.rfo_overlap_npoints.restype = C.c_int32
        L.rfo_baseline_shinozuka.argtypes = [P(Request), C.c_int64, C.c_int64, C.c_int32, C.c_int32, P(d), C.c_int32]
        L.rfo_baseline_shinozuka.restype = d
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleRequest:
    """One generation request; field names follow the reference's RF type."""

    def __init__(self, xPoints, corrMod=CM_GAUSSIAN, margiFirst=FOM_GAUSSIAN, corrL=(1.0, 1.0, 1.0),
                 fieldAvg=0.0, fieldVar=1.0, Nmc=1, method=SHINOZUKA, seedStart=0, kNStep=(0, 0, 0),
                 isoNRadial=0, isoNDir=0, literal=False, normalize=False, xRange=(0.0, 0.0, 0.0)):
        x = np.ascontiguousarray(np.asarray(xPoints, dtype=np.float64))
        if x.ndim == 1:
            x = x.reshape(-1, 1)
        # xPoints is nDim x n in Fortran order == n x nDim in C order
        self.x = x
        self.nDim = x.shape[1]
        self.n = x.shape[0]
        r = Request()
        r.nDim = self.nDim
        r.n = self.n
        r.xPoints = _dptr(self.x)
        r.corrMod = corrMod
        r.margiFirst = margiFirst
        for i in range(3):
            r.corrL[i] = float(corrL[i]) if i < len(corrL) else 1.0
            r.kNStep[i] = int(kNStep[i]) if i < len(kNStep) else 0
            r.xRange[i] = float(xRange[i]) if i < len(xRange) else 0.0
        r.fieldAvg = fieldAvg
        r.fieldVar = fieldVar
        r.Nmc = Nmc
        r.method = method
        r.seedStart = seedStart
        r.isoNRadial = isoNRadial
        r.isoNDir = isoNDir
        r.literal = int(bool(literal))
        r.normalize = int(bool(normalize))
        self.req = r

    def geometry(self) -> Geometry:
        g = Geometry()
        rc = lib().rfo_geometry_of(C.byref(self.req), C.byref(g))
        if rc:
            raise ValueError(f"oracle rejected the request (rc={rc})")
        return g

    def kpoints(self):
        g = self.geometry()
        kp = np.zeros((g.K, self.nDim))
        amp = np.zeros(g.K)
        S = np.zeros(g.K)
        rc = lib().rfo_kpoints(C.byref(self.req), _dptr(kp), _dptr(amp), _dptr(S))
        if rc:
            raise ValueError(rc)
        return kp, amp, S

    def phase_matrix(self):
        g = self.geometry()
        Bc = np.zeros((self.req.Nmc, g.K))
        Bs = np.zeros((self.req.Nmc, g.K))
        rc = lib().rfo_phase_matrix(C.byref(self.req), _dptr(Bc), _dptr(Bs))
        if rc:
            raise ValueError(rc)
        return Bc, Bs  # [r, k]

    def generate(self, rows=None, nthreads=0, recast=False):
        """Field (nrows x Nmc, column-major in memory: returned as [r, i])."""
        nrows = self.n if rows is None else len(rows)
        out = np.zeros((self.req.Nmc, nrows))
        rp = None
        if rows is not None:
            rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64))
            rp = rows.ctypes.data_as(C.POINTER(C.c_int64))
        fn = lib().rfo_generate_recast if recast else lib().rfo_generate
        rc = fn(C.byref(self.req), rp, nrows, _dptr(out), nthreads)
        if rc:
            raise ValueError(f"oracle rejected the request (rc={rc})")
        return out

    def baseline(self, row0, nrows, r0, nr, nthreads=0):
        out = np.zeros((nr, nrows))
        t = lib().rfo_baseline_shinozuka(C.byref(self.req), row0, nrows, r0, nr, _dptr(out), nthreads)
        if t < 0:
            raise ValueError("baseline rejected the request")
        return out, t


def rng(seedStart=None) -> RNG:
    r = RNG()
    if seedStart is None:
        lib().rfo_rng_initialize(C.byref(r))
    else:
        if lib().rfo_rng_seed(C.byref(r), seedStart):
            raise ValueError(seedStart)
    return r


def i4_stream(seedStart, count):
    """The first `count` i4_uni values of generator 1 seeded from seedStart,
    drawn one call after another (rnglib.f90:548-659)."""
    r = rng(seedStart)
    out = np.zeros(int(count), dtype=np.int32)
    lib().rfo_rng_i4_stream(C.byref(r), int(count), out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out


def grid(xMin, xStep, xNStep):
    """setGrid (axis 1 fastest): returns n x nDim."""
    nd = len(xNStep)
    n = int(np.prod(xNStep))
    out = np.zeros((n, nd))
    a = np.asarray(xMin, dtype=np.float64)
    b = np.asarray(xStep, dtype=np.float64)
    c = np.asarray(xNStep, dtype=np.int32)
    lib().rfo_set_grid(nd, _dptr(a), _dptr(b), c.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(out))
    return out


def unity_partition(xNStep, overlapNPoints, faceMask=0xFFFFFFFF):
    nd = len(xNStep)
    a = np.asarray(xNStep, dtype=np.int32)
    b = np.asarray(overlapNPoints, dtype=np.int32)
    out = np.zeros(int(np.prod(xNStep)))
    lib().rfo_unity_partition(nd, a.ctypes.data_as(C.POINTER(C.c_int32)), b.ctypes.data_as(C.POINTER(C.c_int32)),
                              faceMask, _dptr(out))
    return out


def field_statistics(field, xNStep=None, xStep=None):
    """statistics_RF.f90 restated in FP64 with numpy's FFT, step by step.

    field: n x Nmc (point index fastest within a realization).
    Moments by event and global (calculate_average_and_stdVar_MPI,
    statistics_RF.f90:62-63, :80-86).  With xNStep (axis 1 fastest): the
    directional correlation of realization 1 as rebuild_Sk_FFT computes it
    (:275 normalise by the global mean and deviation, forward FFT along the
    axis, :350 divide by N, :360 times the conjugate, :380 mean over the
    other axes, :395 unnormalised backward FFT, :405 real part), lags
    0 .. N/2 - 1 as rebuild_Sk keeps them (:207), and the correlation length
    of rebuild_corrL (:435).
    """
    f = np.asarray(field, dtype=np.float64)
    n, Nmc = f.shape
    S = f.sum(axis=0)
    Q = (f * f).sum(axis=0)
    evnt_avg = S / n
    evnt_std = np.sqrt(Q / n - evnt_avg ** 2)
    gavg = S.sum() / (n * Nmc)
    gstd = np.sqrt(Q.sum() / (n * Nmc) - gavg ** 2)
    out = {"evnt_avg": evnt_avg, "evnt_std": evnt_std, "global_avg": gavg, "global_std": gstd}
    if xNStep is None:
        return out
    nd = len(xNStep)
    a = ((f[:, 0] - gavg) / gstd).reshape(tuple(int(v) for v in reversed(xNStep)))  # a[i_nd, ..., i_1]
    sk, cl = [], []
    for d in range(nd):
        ax = nd - 1 - d
        N = int(xNStep[d])
        F = np.fft.fft(a, axis=ax) / N
        P = F * np.conj(F)
        other = tuple(i for i in range(nd) if i != ax)
        v = P.mean(axis=other) if other else P
        R = (np.fft.ifft(v) * N).real[: N // 2]
        sk.append(R)
        if xStep is not None:
            cl.append(2.0 * (R.sum() - (R[0] + R[-1]) / 2.0) * xStep[d])
    out["sk"] = sk
    if xStep is not None:
        out["corrL"] = np.array(cl)
    return out


def circular_autocorrelation(field_col, xNStep):
    """The same lags by the direct sum the device computes:
    R(l) = mean over the lines along the axis of (1/N) sum_z g(z) g(z+l mod N)."""
    nd = len(xNStep)
    a = np.asarray(field_col, dtype=np.float64).reshape(tuple(int(v) for v in reversed(xNStep)))
    out = []
    for d in range(nd):
        ax = nd - 1 - d
        N = int(xNStep[d])
        R = np.array([(a * np.roll(a, -l, axis=ax)).mean() for l in range(N // 2)])
        out.append(R)
    return out


PI_REF = 3.1415926535898  # constants_RF.f90: PI as the reference writes it


def fft_method_field(xNStep, xStep, corrL, seedStart, corrMod=CM_GAUSSIAN):
    """gen_Std_Gauss_FFT (randomFieldND.f90:520-763) restated with numpy and
    scipy's DCT, single process, one realization; returns the standard
    (pre-marginal) field on the grid, axis 1 fastest.

    Coordinates and steps divided by corrL (gen_Std_Gauss :58-73); k grid of
    set_kPoints' FFT branch (spectra_RF.f90:135-160): kNStep = grid points,
    kDelta = 2 PI / (1.1 xRange), from 0, axis 1 fastest; S of set_SkVec
    (:202-208 Gaussian, :210-220 cm_COS); draws :674-686 (gamma: K draws,
    K - 1 skipped, phi: K draws); X = (gamma - 1/2) sqrt(S) cos(2 PI phi)
    (:695-696); FFTW REDFT01 on every axis = scipy's DCT type 3, norm None
    (:712-733); scale sqrt(prod xStep) in 2-D, 2 sqrt(prod xStep) in 3-D.
    """
    from scipy import fft as sfft

    n = [int(v) for v in xNStep]
    nd = len(n)
    h = np.asarray(xStep, dtype=np.float64) / np.asarray(corrL, dtype=np.float64)[:nd]
    xr = (np.asarray(n) - 1) * h
    kd = 2.0 * PI_REF / (1.1 * xr)
    K = int(np.prod(n))
    r = rng(seedStart)
    u = np.array([lib().rfo_rng_r8_uni_01(C.byref(r)) for _ in range(3 * K - 1)])
    gamma, phi = u[:K], u[2 * K - 1:3 * K - 1]
    idx = np.indices(tuple(reversed(n))).reshape(nd, -1)[::-1]  # idx[d] = i_d, axis 1 fastest
    S = np.ones(K)
    for d in range(nd):
        k = 0.0 + kd[d] * idx[d]
        S = S * 1.0 * np.exp(-((k * k) * 1.0) / (4.0 * PI_REF))
    if corrMod == CM_COS:
        S = np.zeros(K)
        S[5] = 1.0
    X = (gamma - 0.5) * np.sqrt(S) * np.cos(2.0 * PI_REF * phi)
    Y = sfft.dctn(X.reshape(tuple(reversed(n))), type=3, norm=None)
    scale = (2.0 if nd == 3 else 1.0) * np.sqrt(np.prod(h))
    return Y.reshape(-1) * scale


def separable_field(xMin, xStep, xNStep, corrL, Nmc, kNStep=(0, 0, 0), seedStart=0, corrMod=CM_GAUSSIAN):
    """The Shinozuka field on the structured grid xMin + j xStep (axis 1
    fastest) from the oracle's own wavevectors and phases, evaluated axis by
    axis with complex matrix products (FP64): the whole field of a large grid
    in seconds, for full-field comparisons.  Returns [r, i] before the
    marginal map.  Pinned against the oracle's point-by-point sum in
    tests/test_full_field.py.  Test infrastructure: the checker of the
    whole-field comparisons, never the thing measured."""
    nd = len(xNStep)
    xr = tuple((xNStep[d] - 1) * xStep[d] for d in range(nd))
    req = OracleRequest(np.asarray(xMin, dtype=np.float64).reshape(1, nd), corrL=corrL, Nmc=Nmc, kNStep=kNStep,
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
