"""B200-native spectral-sum random-field generator (randomFieldND path of
cottereau/randomField) behind a C-ABI.

The Python layer is a thin ctypes mirror of the reference interface
``createStandardGaussianFieldUnstruct(xPoints, corrMod, margiFirst, corrL,
fieldAvg, fieldVar, Nmc, method, randField)`` (README.md:58-92): the same
argument names, meanings and layouts (xPoints nDim x n, randField n x Nmc,
Fortran column-major), strings or integer ids for corrMod/margiFirst, and
the reference's error rules raised as :class:`RandomFieldError` instead of
``stop``/``MPI_ABORT``.  All computation happens in librf_b200.so on the GPU;
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = [
    "RandomFieldError", "Options", "Context", "lib", "create_standard_gaussian_field_unstruct",
    "query_geometry", "generate_device_noalloc", "Request", "BatchStats", "make_request", "generate_batch",
    "Server", "ServerConfig", "ServerStats", "BlendGrid", "blend_layout", "ISOTROPIC", "RANDOMIZATION", "SHINOZUKA", "CM_GAUSSIAN", "CM_COS", "FOM_GAUSSIAN", "FOM_LOGNORMAL",
    "PREC_BF16", "PREC_FP16", "PREC_FP32", "PREC_BF16_FAST", "PREC_FP8", "LIB_PATH", "STATUS",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librf_b200.so")

# constants_RF.f90:12-21
ISOTROPIC, SHINOZUKA, RANDOMIZATION, FFT = 1, 2, 3, 4
CM_GAUSSIAN, CM_COS = 1, 2
FOM_GAUSSIAN, FOM_LOGNORMAL = 1, 2
PREC_BF16, PREC_FP16, PREC_FP32, PREC_BF16_FAST, PREC_FP8 = 0, 1, 2, 3, 4

STATUS = {
    0: "RF_OK", -1: "RF_EINVAL_NMC", -2: "RF_EINVAL_NDIM", -3: "RF_EINVAL_CORRL", -4: "RF_EINVAL_LOGNORMAL",
    -5: "RF_EINVAL_METHOD", -6: "RF_EINVAL_CORRMOD", -7: "RF_EINVAL_MARGINAL", -8: "RF_EINVAL_RANGE",
    -9: "RF_EINVAL_ARG", -10: "RF_ENOTSUP", -20: "RF_ECUDA", -21: "RF_ENOMEM", -22: "RF_ETIMEDOUT",
    -23: "RF_ENOMEM_ADMISSION", -24: "RF_ESCRATCH", -25: "RF_ENODEV", -26: "RF_EBOUNDS",
}

_CORRMOD = {"gaussian": CM_GAUSSIAN, "cos": CM_COS, "cm_gaussian": CM_GAUSSIAN, "cm_cos": CM_COS}
_MARGI = {"gaussian": FOM_GAUSSIAN, "lognormal": FOM_LOGNORMAL}
_PREC = {"bf16": PREC_BF16, "fp16": PREC_FP16, "fp32": PREC_FP32, "bf16_fast": PREC_BF16_FAST, "fp8": PREC_FP8}

# Every symbol include/randomfield_b200.h declares.
EXPORTS = [
    "rf_options_init", "rf_create_standard_gaussian_field_unstruct", "rf_context_create", "rf_context_destroy",
    "rf_generate_device", "rf_context_synchronize", "rf_query_geometry", "rf_last_error", "rf_abi_version",
    "rf_context_set_timing", "rf_context_last_times", "rf_generate_device_noalloc",
    "rf_generate_batch", "rf_generate_batch_device", "rf_batch_last_stats",
    "rf_server_config_init", "rf_server_create", "rf_server_submit", "rf_server_wait", "rf_server_get_stats",
    "rf_server_destroy", "rf_server_submit_blended", "rf_context_selftest_timeout", "rf_measure_sfu_rate", "rf_blend_layout", "rf_generate_blended", "rf_generate_blended_device",
    "rf_field_statistics", "rf_generate_fft_grid", "rf_generate_grid", "rf_create_standard_gaussian_field_grid",
    "rf_write_result_grid", "rf_debug_table_draws", "rf_context_selftest_bounds", "rf_debug_bounds_build",
]


class RandomFieldError(RuntimeError):
    """A non-zero status of the C-ABI (the reference would stop or abort)."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.status = STATUS.get(code, str(code))
        super().__init__(f"{self.status} ({code}): {message}")


class Options(C.Structure):
    """rf_options (include/randomfield_b200.h)."""

    _fields_ = [
        ("size", C.c_int32),
        ("precision", C.c_int32),
        ("seed_start", C.c_int64),
        ("k_nstep", C.c_int32 * 3),
        ("iso_n_radial", C.c_int32),
        ("iso_n_dir", C.c_int32),
        ("literal", C.c_int32),
        ("normalize", C.c_int32),
        ("x_range", C.c_double * 3),
        ("device", C.c_int32),
        ("reserved0", C.c_int32),
        ("draws", C.c_void_p),
        ("n_draws", C.c_int64),
        ("reserved", C.c_int32 * 2),
    ]

    @classmethod
    def make(cls, precision="bf16", seed_start=0, k_nstep=(0, 0, 0), iso_n_radial=0, iso_n_dir=0,
             literal=False, normalize=False, x_range=(0.0, 0.0, 0.0), device=0, draws=None) -> "Options":
        """``draws``: optional float64 uniform draws in [0, 1) replacing the
        rnglib stream, in the reference's order of random_number calls (see
        rf_options.draws); the array must stay alive while the call runs."""
        o = cls()
        lib().rf_options_init(C.byref(o))
        o.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
        o.seed_start = int(seed_start)
        for i in range(3):
            o.k_nstep[i] = int(k_nstep[i]) if i < len(k_nstep) else 0
            o.x_range[i] = float(x_range[i]) if i < len(x_range) else 0.0
        o.iso_n_radial = int(iso_n_radial)
        o.iso_n_dir = int(iso_n_dir)
        o.literal = int(bool(literal))
        o.normalize = int(bool(normalize))
        o.device = int(device)
        if draws is not None:
            d = np.ascontiguousarray(np.asarray(draws, dtype=np.float64).reshape(-1))
            o._draws_keep = d  # the struct points into it
            o.draws = d.ctypes.data
            o.n_draws = int(d.size)
        return o


class Request(C.Structure):
    """rf_request (include/randomfield_b200.h): one request of a batch."""

    _fields_ = [
        ("xPoints", C.c_void_p),
        ("randField", C.c_void_p),
        ("n", C.c_int64),
        ("nDim", C.c_int32),
        ("corrMod", C.c_int32),
        ("margiFirst", C.c_int32),
        ("Nmc", C.c_int32),
        ("method", C.c_int32),
        ("reserved0", C.c_int32),
        ("corrL", C.c_double * 3),
        ("fieldAvg", C.c_double),
        ("fieldVar", C.c_double),
        ("opt", Options),
    ]


class FieldStats(C.Structure):
    """rf_field_stats: global moments of a field (statistics_RF.f90:18-174)."""

    _fields_ = [
        ("global_avg", C.c_double),
        ("global_std", C.c_double),
        ("n", C.c_int64),
        ("Nmc", C.c_int32),
        ("nDim", C.c_int32),
    ]


class BatchStats(C.Structure):
    """rf_batch_stats: the last grouped launch of a context."""

    _fields_ = [
        ("tables_ms", C.c_double),
        ("contract_ms", C.c_double),
        ("units", C.c_int64),
        ("work_items", C.c_int64),
        ("realization_block", C.c_int32),
        ("stages", C.c_int32),
        ("graph_replayed", C.c_int32),
        ("tuned", C.c_int32),
        ("outer_stages", C.c_int32),
        ("tune_candidates", C.c_int32),
        ("tune_default_ms", C.c_double),
        ("tune_best_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BlendGrid(C.Structure):
    """rf_blend_grid: a structured group grid split into overlapping subdomains."""

    _fields_ = [
        ("nDim", C.c_int32),
        ("xNStep", C.c_int32 * 3),
        ("nFields", C.c_int32 * 3),
        ("reserved0", C.c_int32),
        ("xMin", C.c_double * 3),
        ("xStep", C.c_double * 3),
        ("overlap", C.c_double),
        ("reserved", C.c_int32 * 8),
    ]

    @classmethod
    def make(cls, xNStep, xStep, nFields, overlap, xMin=None) -> "BlendGrid":
        g = cls()
        nd = len(xNStep)
        g.nDim = nd
        for d in range(3):
            g.xNStep[d] = int(xNStep[d]) if d < nd else 1
            g.nFields[d] = int(nFields[d]) if d < nd else 1
            g.xStep[d] = float(xStep[d]) if d < nd else 0.0
            g.xMin[d] = float(xMin[d]) if (xMin is not None and d < nd) else 0.0
        g.overlap = float(overlap)
        return g


def blend_layout(grid: "BlendGrid", corrL):
    """(subdomain points per axis, overlapNPoints per axis) of a blend grid."""
    cl = np.ascontiguousarray(np.asarray(list(corrL) + [1.0] * (3 - len(corrL)), dtype=np.float64))
    L = (C.c_int32 * 3)()
    O = (C.c_int32 * 3)()
    _check(lib().rf_blend_layout(C.byref(grid), cl.ctypes.data_as(C.POINTER(C.c_double)), L, O))
    return list(L), list(O)


class ServerConfig(C.Structure):
    """rf_server_config."""

    _fields_ = [
        ("size", C.c_int32),
        ("device", C.c_int32),
        ("precision", C.c_int32),
        ("max_batch", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("reserved", C.c_int32 * 8),
    ]


class ServerStats(C.Structure):
    """rf_server_stats."""

    _fields_ = [
        ("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("batches", C.c_int64),
        ("admission_waits", C.c_int64), ("peak_bytes", C.c_int64), ("field_values", C.c_double),
        ("busy_ms", C.c_double), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
        ("mean_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    """The loaded librf_b200.so (raises if it was not built).  RF_LIB names
    another build of the same library to load instead (the index-checked
    librf_b200_bounds.so of `python -m randomfield_b200.build --debug-bounds`)."""
    global _lib
    if _lib is None:
        path = os.environ.get("RF_LIB") or LIB_PATH
        if not os.path.exists(path):
            raise RandomFieldError(-25, f"{path} is missing: run `python -m randomfield_b200.build`")
        L = C.CDLL(path)
        P, d, i32, i64 = C.POINTER, C.c_double, C.c_int, C.c_int64
        L.rf_options_init.argtypes = [P(Options)]
        L.rf_options_init.restype = None
        L.rf_last_error.restype = C.c_char_p
        L.rf_abi_version.restype = C.c_int
        L.rf_create_standard_gaussian_field_unstruct.argtypes = [
            P(d), i32, i64, i32, i32, P(d), d, d, i32, i32, P(d), P(Options)]
        L.rf_context_create.argtypes = [i32, P(C.c_void_p)]
        L.rf_context_destroy.argtypes = [C.c_void_p]
        L.rf_context_synchronize.argtypes = [C.c_void_p]
        L.rf_context_set_timing.argtypes = [C.c_void_p, i32]
        L.rf_context_last_times.argtypes = [C.c_void_p, P(d), P(d), P(d), P(C.c_int32)]
        L.rf_generate_device.argtypes = [C.c_void_p, C.c_void_p, i32, i64, i32, i32, P(d), d, d, i32, i32,
                                         C.c_void_p, P(Options), C.c_void_p]
        L.rf_generate_device_noalloc.argtypes = [C.c_void_p, i32, i64, i32, i32, P(d), d, d, i32, i32, C.c_void_p,
                                                 P(Options), C.c_void_p]
        L.rf_query_geometry.argtypes = [P(d), i32, i64, i32, P(d), i32, P(Options), P(i64), P(C.c_int32), P(d),
                                        P(d)]
        L.rf_generate_batch.argtypes = [C.c_void_p, P(Request), C.c_int32]
        L.rf_generate_batch_device.argtypes = [C.c_void_p, P(Request), C.c_int32, C.c_void_p]
        L.rf_batch_last_stats.argtypes = [C.c_void_p, P(BatchStats)]
        L.rf_server_config_init.argtypes = [P(ServerConfig)]
        L.rf_server_config_init.restype = None
        L.rf_server_create.argtypes = [P(ServerConfig), P(C.c_void_p)]
        L.rf_server_submit.argtypes = [C.c_void_p, P(Request), P(i64)]
        L.rf_server_wait.argtypes = [C.c_void_p, i64, d, P(d)]
        L.rf_server_get_stats.argtypes = [C.c_void_p, P(ServerStats)]
        L.rf_server_destroy.argtypes = [C.c_void_p]
        L.rf_context_selftest_timeout.argtypes = [C.c_void_p, d]
        L.rf_measure_sfu_rate.argtypes = [i32, P(d)]
        L.rf_debug_table_draws.argtypes = [i32, i32, i32, P(Options), P(i64), P(i32), i64, P(i32), i64]
        L.rf_context_selftest_bounds.argtypes = [C.c_void_p]
        L.rf_debug_bounds_build.argtypes = []
        L.rf_generate_fft_grid.argtypes = [C.c_void_p, i32, P(i64), P(d), i32, i32, P(d), d, d, i32, C.c_void_p,
                                           P(Options)]
        L.rf_generate_grid.argtypes = [C.c_void_p, i32, P(d), P(d), P(i64), i32, i32, P(d), d, d, i32, i32,
                                       C.c_void_p, P(Options), C.c_void_p]
        L.rf_write_result_grid.argtypes = [C.c_char_p, C.c_char_p, i32, P(d), P(d), P(d), P(d),
                                           C.POINTER(ResultAttributes)]
        L.rf_create_standard_gaussian_field_grid.argtypes = [i32, P(d), P(d), P(i64), i32, i32, P(d), d, d, i32, i32,
                                                             P(d), P(Options)]
        L.rf_field_statistics.argtypes = [C.c_void_p, C.c_void_p, i64, i32, i32, P(i64), P(d), P(d), P(d), P(d),
                                          P(d), P(FieldStats)]
        L.rf_blend_layout.argtypes = [P(BlendGrid), P(d), P(C.c_int32), P(C.c_int32)]
        L.rf_server_submit_blended.argtypes = [C.c_void_p, P(BlendGrid), i32, i32, P(d), d, d, i32, i32, P(d),
                                               P(Options), P(i64)]
        L.rf_generate_blended.argtypes = [C.c_void_p, P(BlendGrid), i32, i32, P(d), d, d, i32, i32, P(d),
                                          P(Options)]
        L.rf_generate_blended_device.argtypes = [C.c_void_p, P(BlendGrid), i32, i32, P(d), d, d, i32, i32,
                                                 C.c_void_p, P(Options), C.c_void_p]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RandomFieldError(rc, lib().rf_last_error().decode())


def _id(v, table, what):
    if isinstance(v, str):
        key = v.strip().lower()
        if key not in table:
            raise RandomFieldError(-9, f"unknown {what} '{v}'")
        return table[key]
    return int(v)


def _points(xPoints) -> np.ndarray:
    """xPoints as nDim x n (reference layout) -> Fortran-ordered float64."""
    x = np.asarray(xPoints, dtype=np.float64)
    if x.ndim == 1:
        x = x.reshape(1, -1)
    return np.asfortranarray(x)


def _opts(opts) -> Options:
    if opts is None:
        return Options.make()
    if isinstance(opts, Options):
        return opts
    return Options.make(**opts)


def create_standard_gaussian_field_unstruct(xPoints, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method,
                                            randField=None, options=None, **kw):
    """Generate Nmc realizations at the points; returns randField (n x Nmc).

    Mirrors createStandardGaussianFieldUnstruct (README.md:58-92).  ``xPoints``
    is nDim x n; ``randField``, if given, must be a Fortran-ordered float64
    n x Nmc array and is filled in place.  Extra keywords build an
    :class:`Options` (precision, seed_start, k_nstep, iso_n_radial, iso_n_dir,
    literal, normalize, x_range, device).
    """
    x = _points(xPoints)
    nDim, n = x.shape
    cm = _id(corrMod, _CORRMOD, "corrMod")
    mf = _id(margiFirst, _MARGI, "margiFirst")
    cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
    if cl.size < nDim:
        raise RandomFieldError(-9, f"corrL needs {nDim} entries")
    if randField is None:
        randField = np.empty((n, int(Nmc)), dtype=np.float64, order="F")
    elif (randField.dtype != np.float64 or not randField.flags.f_contiguous
          or randField.shape != (n, int(Nmc))):
        raise RandomFieldError(-9, "randField must be a Fortran-ordered float64 n x Nmc array")
    o = _opts(options if options is not None else (kw or None))
    P = C.POINTER(C.c_double)
    _check(lib().rf_create_standard_gaussian_field_unstruct(
        x.ctypes.data_as(P), nDim, n, cm, mf, cl.ctypes.data_as(P), float(fieldAvg), float(fieldVar), int(Nmc),
        int(method), randField.ctypes.data_as(P), C.byref(o)))
    return randField


class ResultAttributes(C.Structure):
    """rf_result_attributes: the run parameters written on a result file
    (write_HDF5_attributes, writeResultFile_RF.f90:1758-1849)."""

    _fields_ = [(nm, C.c_int32) for nm in ("nb_procs", "nDim", "Nmc", "method", "seedStart", "corrMod",
                                           "margiFirst", "localizationLevel")] + [
        ("kNStep", C.c_int32 * 3), ("nFields", C.c_int32 * 3)] + [
        (nm, C.c_double * 3) for nm in ("xMinGlob", "xMaxGlob", "xStep", "corrL", "overlap", "procExtent",
                                        "kMax_out")]

    @classmethod
    def make(cls, **kw) -> "ResultAttributes":
        a = cls()
        for k, v in kw.items():
            f = getattr(a, k)
            if isinstance(f, (int, float)):
                setattr(a, k, v)
            else:
                for i, x in enumerate(v):
                    f[i] = x
        return a


def write_result_grid(folder, fileName, xMin, xMax, xStep, field, attributes=None) -> None:
    """rf_write_result_grid: <folder>/h5/<fileName>.h5 (dataset "samples",
    one realization on the structured grid, attributes from a dict or a
    ResultAttributes) and, in 2-D and 3-D, <folder>/xmf/<fileName>.xmf."""
    nDim = len(xMin)
    P = C.POINTER(C.c_double)
    a = np.ascontiguousarray(np.asarray(xMin, dtype=np.float64).reshape(-1))
    b = np.ascontiguousarray(np.asarray(xMax, dtype=np.float64).reshape(-1))
    h = np.ascontiguousarray(np.asarray(xStep, dtype=np.float64).reshape(-1))
    f = np.ascontiguousarray(np.asarray(field, dtype=np.float64).reshape(-1))
    if np.all(h > 0):  # otherwise the library reports the bad step
        n = 1
        for d in range(nDim):
            n *= int(round((b[d] - a[d]) / h[d])) + 1
        if f.size != n:
            raise RandomFieldError(-9, f"field has {f.size} values, the grid {n}")
    at = attributes
    if isinstance(at, dict):
        at = ResultAttributes.make(**at)
    _check(lib().rf_write_result_grid(str(folder).encode(), str(fileName).encode(), int(nDim), a.ctypes.data_as(P),
                                      b.ctypes.data_as(P), h.ctypes.data_as(P), f.ctypes.data_as(P),
                                      C.byref(at) if at is not None else None))


def create_standard_gaussian_field_grid(xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc,
                                        method=SHINOZUKA, randField=None, options=None, **kw):
    """rf_create_standard_gaussian_field_grid: the Shinozuka field on the
    structured grid xMin + j * xStep (xNStep points per axis, axis 1
    fastest), evaluated axis by axis in FP64; returns randField
    (prod(xNStep) x Nmc, Fortran-ordered), filled in place if given."""
    nDim = len(xNStep)
    a = np.ascontiguousarray(np.asarray(xMin, dtype=np.float64).reshape(-1))
    h = np.ascontiguousarray(np.asarray(xStep, dtype=np.float64).reshape(-1))
    g = np.ascontiguousarray(np.asarray(xNStep, dtype=np.int64).reshape(-1))
    cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
    if not (len(a) == len(h) == len(cl) == nDim):
        raise RandomFieldError(-9, "xMin, xStep, xNStep and corrL need one entry per axis")
    n = int(np.prod(g))
    if randField is None:
        randField = np.empty((n, int(Nmc)), dtype=np.float64, order="F")
    elif (randField.dtype != np.float64 or not randField.flags.f_contiguous
          or randField.shape != (n, int(Nmc))):
        raise RandomFieldError(-9, "randField must be a Fortran-ordered float64 n x Nmc array")
    o = _opts(options if options is not None else (kw or None))
    P = C.POINTER(C.c_double)
    _check(lib().rf_create_standard_gaussian_field_grid(
        int(nDim), a.ctypes.data_as(P), h.ctypes.data_as(P), g.ctypes.data_as(C.POINTER(C.c_int64)),
        _id(corrMod, _CORRMOD, "corrMod"), _id(margiFirst, _MARGI, "margiFirst"), cl.ctypes.data_as(P),
        float(fieldAvg), float(fieldVar), int(Nmc), int(method), randField.ctypes.data_as(P), C.byref(o)))
    return randField


def query_geometry(xPoints, corrMod, corrL, method, options=None, **kw):
    """(K, kNStep[3], kDelta[3], ampMult) exactly as the generator uses them."""
    x = _points(xPoints)
    nDim, n = x.shape
    cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
    o = _opts(options if options is not None else (kw or None))
    K = C.c_int64()
    kn = (C.c_int32 * 3)()
    kd = (C.c_double * 3)()
    am = C.c_double()
    P = C.POINTER(C.c_double)
    _check(lib().rf_query_geometry(x.ctypes.data_as(P), nDim, n, _id(corrMod, _CORRMOD, "corrMod"),
                                   cl.ctypes.data_as(P), int(method), C.byref(o), C.byref(K), kn, kd,
                                   C.byref(am)))
    return K.value, list(kn), list(kd), am.value


def generate_device_noalloc(d_x, nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, d_out,
                            options=None, stream=0, **kw) -> None:
    """rf_generate_device_noalloc: device buffers in, field out, no device
    allocation by the library (a fixed 32 MiB scratch array per GPU instead);
    for callers whose allocator owns device memory.  Returns when done."""
    cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
    o = _opts(options if options is not None else (kw or None))
    s = stream if isinstance(stream, int) else int(getattr(stream, "cuda_stream", 0))
    ptr = Context._ptr
    _check(lib().rf_generate_device_noalloc(C.c_void_p(ptr(d_x)), int(nDim), int(n), _id(corrMod, _CORRMOD, "corrMod"),
                                            _id(margiFirst, _MARGI, "margiFirst"),
                                            cl.ctypes.data_as(C.POINTER(C.c_double)), float(fieldAvg), float(fieldVar),
                                            int(Nmc), int(method), C.c_void_p(ptr(d_out)), C.byref(o), C.c_void_p(s)))


def measure_sfu_rate(device: int = 0) -> float:
    """MUFU (sin, cos) pairs per second of the device (rf_measure_sfu_rate)."""
    v = C.c_double()
    _check(lib().rf_measure_sfu_rate(int(device), C.byref(v)))
    return v.value


def debug_table_draws(nDim, method, Nmc, options=None, **kw):
    """rf_debug_table_draws: the i4_uni draws the device table builder
    consumes, in reference order.  Returns (draws, k_draws): draws is
    [Nmc, K] (the phase draw) or [Nmc, K, 2] for the isotropic method (gamma,
    psi); k_draws is [K, 2] (theta, phi) for the isotropic method, else None.
    The options must fix the wavevector count (k_nstep / iso_n_radial, or
    x_range)."""
    o = _opts(options if options is not None else (kw or None))
    K = C.c_int64()
    _check(lib().rf_debug_table_draws(int(nDim), int(method), int(Nmc), C.byref(o), C.byref(K), None, 0, None, 0))
    D = 2 if int(method) == ISOTROPIC else 1
    draws = np.zeros(int(Nmc) * K.value * D, dtype=np.int32)
    kd = np.zeros(2 * K.value, dtype=np.int32) if int(method) == ISOTROPIC else None
    P32 = C.POINTER(C.c_int32)
    _check(lib().rf_debug_table_draws(int(nDim), int(method), int(Nmc), C.byref(o), C.byref(K),
                                      draws.ctypes.data_as(P32), draws.size,
                                      kd.ctypes.data_as(P32) if kd is not None else None,
                                      kd.size if kd is not None else 0))
    shape = (int(Nmc), K.value, 2) if D == 2 else (int(Nmc), K.value)
    return draws.reshape(shape), (kd.reshape(K.value, 2) if kd is not None else None)


def make_request(xPoints, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, randField,
                 options=None, **kw) -> Request:
    """An rf_request over buffers the caller keeps alive until the batch
    returns: ``xPoints``/``randField`` are device pointers (ints or objects
    with ``data_ptr()``) for the device batch, or numpy arrays (nDim x n and
    Fortran-ordered n x Nmc float64) for the host batch."""
    r = Request()
    if isinstance(xPoints, np.ndarray):
        if xPoints.dtype != np.float64 or not xPoints.flags.f_contiguous:
            raise RandomFieldError(-9, "xPoints must be a Fortran-ordered float64 nDim x n array")
        nDim, n = xPoints.shape
        if (randField.dtype != np.float64 or not randField.flags.f_contiguous
                or randField.shape != (n, int(Nmc))):
            raise RandomFieldError(-9, "randField must be a Fortran-ordered float64 n x Nmc array")
        r.xPoints, r.randField = xPoints.ctypes.data, randField.ctypes.data
    else:
        nDim, n = kw.pop("nDim"), kw.pop("n")
        r.xPoints, r.randField = Context._ptr(xPoints), Context._ptr(randField)
    r.n, r.nDim = int(n), int(nDim)
    r.corrMod = _id(corrMod, _CORRMOD, "corrMod")
    r.margiFirst = _id(margiFirst, _MARGI, "margiFirst")
    cl = list(np.asarray(corrL, dtype=np.float64).reshape(-1))
    for i in range(3):
        r.corrL[i] = float(cl[i]) if i < len(cl) else 1.0
    r.fieldAvg, r.fieldVar = float(fieldAvg), float(fieldVar)
    r.Nmc, r.method = int(Nmc), int(method)
    r.opt = _opts(options if options is not None else (kw or None))
    return r


def generate_batch(ctx: "Context", requests) -> None:
    """rf_generate_batch: host-buffer requests (see :func:`make_request`),
    one grouped launch; returns when every randField is filled."""
    arr = (Request * len(requests))(*requests)
    _check(lib().rf_generate_batch(ctx._h, arr, len(requests)))


class Server:
    """rf_server: the serving loop (continuous batching, HBM admission).

    ``submit(request)`` takes a host-buffer :class:`Request` (keep its arrays
    alive until ``wait`` returns) and returns a ticket; ``wait(ticket)``
    returns the request's latency in milliseconds or raises its error.
    """

    def __init__(self, device=0, precision="bf16", max_batch=512, hbm_budget_bytes=0):
        cfg = ServerConfig()
        lib().rf_server_config_init(C.byref(cfg))
        cfg.device = int(device)
        cfg.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
        cfg.max_batch = int(max_batch)
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        h = C.c_void_p()
        _check(lib().rf_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, request: Request, keep=None) -> int:
        t = C.c_int64()
        _check(lib().rf_server_submit(self._h, C.byref(request), C.byref(t)))
        self._keep[t.value] = (request, keep)
        return t.value

    def submit_blended(self, grid: "BlendGrid", corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method,
                       randField, options=None, **kw) -> int:
        """Queues a localization blend; randField is a Fortran-ordered
        float64 (group points x Nmc) array kept alive until ``wait``."""
        cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
        o = _opts(options if options is not None else (kw or None))
        t = C.c_int64()
        P = C.POINTER(C.c_double)
        _check(lib().rf_server_submit_blended(self._h, C.byref(grid), _id(corrMod, _CORRMOD, "corrMod"),
                                              _id(margiFirst, _MARGI, "margiFirst"), cl.ctypes.data_as(P),
                                              float(fieldAvg), float(fieldVar), int(Nmc), int(method),
                                              randField.ctypes.data_as(P), C.byref(o), C.byref(t)))
        self._keep[t.value] = (grid, randField, cl, o)
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0) -> float:
        lat = C.c_double()
        try:
            _check(lib().rf_server_wait(self._h, int(ticket), float(timeout_s), C.byref(lat)))
        finally:
            self._keep.pop(int(ticket), None)
        return lat.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().rf_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().rf_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """rf_context: device-resident generation on a CUDA stream.

    ``generate(d_x, d_out, ...)`` takes device pointers (ints) or objects with
    ``data_ptr()`` (torch tensors): d_x holds nDim x n float64 (point-major),
    d_out n x Nmc float64 column-major.
    """

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().rf_context_create(int(device), C.byref(h)))
        self._h = h
        self.device = int(device)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().rf_context_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(t) -> int:
        return int(t.data_ptr()) if hasattr(t, "data_ptr") else int(t)

    def generate(self, d_x, nDim, n, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, d_out,
                 options=None, stream=0, **kw) -> None:
        cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
        o = _opts(options if options is not None else (kw or None))
        s = stream if isinstance(stream, int) else int(getattr(stream, "cuda_stream", 0))
        _check(lib().rf_generate_device(self._h, C.c_void_p(self._ptr(d_x)), int(nDim), int(n),
                                        _id(corrMod, _CORRMOD, "corrMod"), _id(margiFirst, _MARGI, "margiFirst"),
                                        cl.ctypes.data_as(C.POINTER(C.c_double)), float(fieldAvg), float(fieldVar),
                                        int(Nmc), int(method), C.c_void_p(self._ptr(d_out)), C.byref(o),
                                        C.c_void_p(s)))

    def selftest_bounds(self) -> None:
        """rf_context_selftest_bounds: raises RandomFieldError(RF_EBOUNDS) in
        the RF_DEBUG_BOUNDS build (its index check caught the planted index),
        RF_ENOTSUP in the normal build."""
        _check(lib().rf_context_selftest_bounds(self._h))

    def selftest_timeout(self, limit_ms: float = 50.0) -> None:
        """rf_context_selftest_timeout: raises RandomFieldError(RF_ETIMEDOUT)
        when the bounded device wait expired as designed."""
        _check(lib().rf_context_selftest_timeout(self._h, float(limit_ms)))

    def synchronize(self) -> None:
        _check(lib().rf_context_synchronize(self._h))

    def set_timing(self, enable: bool = True) -> None:
        _check(lib().rf_context_set_timing(self._h, int(bool(enable))))

    def generate_batch_device(self, requests, stream=0) -> None:
        """rf_generate_batch_device: device-buffer requests, queued on the stream."""
        s = stream if isinstance(stream, int) else int(getattr(stream, "cuda_stream", 0))
        arr = (Request * len(requests))(*requests)
        _check(lib().rf_generate_batch_device(self._h, arr, len(requests), C.c_void_p(s)))

    def generate_blended(self, grid: "BlendGrid", corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc, method,
                         randField=None, options=None, **kw):
        """rf_generate_blended: the blended field on the group grid, returned
        (or written into randField) as a Fortran-ordered G x Nmc array."""
        G = int(np.prod([grid.xNStep[d] for d in range(grid.nDim)]))
        if randField is None:
            randField = np.empty((G, int(Nmc)), dtype=np.float64, order="F")
        cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
        o = _opts(options if options is not None else (kw or None))
        P = C.POINTER(C.c_double)
        _check(lib().rf_generate_blended(self._h, C.byref(grid), _id(corrMod, _CORRMOD, "corrMod"),
                                         _id(margiFirst, _MARGI, "margiFirst"), cl.ctypes.data_as(P),
                                         float(fieldAvg), float(fieldVar), int(Nmc), int(method),
                                         randField.ctypes.data_as(P), C.byref(o)))
        return randField

    def generate_blended_device(self, grid: "BlendGrid", corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc,
                                method, d_out, options=None, stream=0, **kw) -> None:
        cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
        o = _opts(options if options is not None else (kw or None))
        s = stream if isinstance(stream, int) else int(getattr(stream, "cuda_stream", 0))
        _check(lib().rf_generate_blended_device(self._h, C.byref(grid), _id(corrMod, _CORRMOD, "corrMod"),
                                                _id(margiFirst, _MARGI, "margiFirst"),
                                                cl.ctypes.data_as(C.POINTER(C.c_double)), float(fieldAvg),
                                                float(fieldVar), int(Nmc), int(method), C.c_void_p(self._ptr(d_out)),
                                                C.byref(o), C.c_void_p(s)))

    def generate_fft_grid(self, d_out, xNStep, xStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc,
                          options=None, **kw) -> None:
        """rf_generate_fft_grid: the FFT method (method 4) on a structured grid
        of xNStep points spaced xStep per axis (2-D or 3-D, axis 1 fastest);
        d_out holds prod(xNStep) x Nmc float64 column-major (e.g. a torch
        tensor of shape (Nmc, prod(xNStep)))."""
        nDim = len(xNStep)
        g = np.ascontiguousarray(np.asarray(xNStep, dtype=np.int64).reshape(-1))
        h = np.ascontiguousarray(np.asarray(xStep, dtype=np.float64).reshape(-1))
        cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
        o = _opts(options if options is not None else (kw or None))
        P = C.POINTER(C.c_double)
        _check(lib().rf_generate_fft_grid(self._h, int(nDim), g.ctypes.data_as(C.POINTER(C.c_int64)), h.ctypes.data_as(P),
                                          _id(corrMod, _CORRMOD, "corrMod"), _id(margiFirst, _MARGI, "margiFirst"),
                                          cl.ctypes.data_as(P), float(fieldAvg), float(fieldVar), int(Nmc),
                                          C.c_void_p(self._ptr(d_out)), C.byref(o)))

    def generate_grid(self, d_out, xMin, xStep, xNStep, corrMod, margiFirst, corrL, fieldAvg, fieldVar, Nmc,
                      method=SHINOZUKA, options=None, stream=0, **kw) -> None:
        """rf_generate_grid: the Shinozuka field on the structured grid
        xMin + j * xStep (xNStep points per axis, axis 1 fastest), evaluated
        axis by axis in FP64; d_out holds prod(xNStep) x Nmc float64
        column-major (e.g. a torch tensor of shape (Nmc, prod(xNStep)))."""
        nDim = len(xNStep)
        a = np.ascontiguousarray(np.asarray(xMin, dtype=np.float64).reshape(-1))
        h = np.ascontiguousarray(np.asarray(xStep, dtype=np.float64).reshape(-1))
        g = np.ascontiguousarray(np.asarray(xNStep, dtype=np.int64).reshape(-1))
        cl = np.ascontiguousarray(np.asarray(corrL, dtype=np.float64).reshape(-1))
        if not (len(a) == len(h) == len(cl) == nDim):
            raise ValueError("xMin, xStep, xNStep and corrL need one entry per axis")
        o = _opts(options if options is not None else (kw or None))
        s = stream if isinstance(stream, int) else int(getattr(stream, "cuda_stream", 0))
        P = C.POINTER(C.c_double)
        _check(lib().rf_generate_grid(self._h, int(nDim), a.ctypes.data_as(P), h.ctypes.data_as(P),
                                      g.ctypes.data_as(C.POINTER(C.c_int64)), _id(corrMod, _CORRMOD, "corrMod"),
                                      _id(margiFirst, _MARGI, "margiFirst"), cl.ctypes.data_as(P), float(fieldAvg),
                                      float(fieldVar), int(Nmc), int(method), C.c_void_p(self._ptr(d_out)),
                                      C.byref(o), C.c_void_p(s)))

    def field_statistics(self, d_field, n: int, Nmc: int, nDim: int = 3, grid=None, step=None) -> dict:
        """rf_field_statistics on a device field (n x Nmc column-major, e.g.
        a torch tensor of shape (Nmc, n)): per-realization mean and standard
        deviation, global mean and deviation, and with ``grid`` (points per
        axis, axis 1 fastest) and ``step`` the directional correlation of
        realization 1 (lags 0 .. N_d/2 - 1 per axis) and the correlation
        length estimate per axis."""
        P = C.POINTER(C.c_double)
        avg = np.empty(int(Nmc))
        std = np.empty(int(Nmc))
        st = FieldStats()
        out = {}
        if grid is not None:
            g = np.ascontiguousarray(np.asarray(grid, dtype=np.int64).reshape(-1)[:nDim])
            h = np.ascontiguousarray(np.asarray(step, dtype=np.float64).reshape(-1)[:nDim]) if step is not None \
                else None
            sk = np.empty(int(sum(int(v) // 2 for v in g)))
            cl = np.empty(int(nDim))
            _check(lib().rf_field_statistics(self._h, C.c_void_p(self._ptr(d_field)), int(n), int(Nmc), int(nDim),
                                             g.ctypes.data_as(C.POINTER(C.c_int64)),
                                             h.ctypes.data_as(P) if h is not None else None, avg.ctypes.data_as(P),
                                             std.ctypes.data_as(P), sk.ctypes.data_as(P),
                                             cl.ctypes.data_as(P) if h is not None else None, C.byref(st)))
            parts, o = [], 0
            for v in g:
                parts.append(sk[o:o + int(v) // 2])
                o += int(v) // 2
            out["sk"] = parts
            if h is not None:
                out["corrL"] = cl
        else:
            _check(lib().rf_field_statistics(self._h, C.c_void_p(self._ptr(d_field)), int(n), int(Nmc), int(nDim),
                                             None, None, avg.ctypes.data_as(P), std.ctypes.data_as(P), None, None,
                                             C.byref(st)))
        out.update(evnt_avg=avg, evnt_std=std, global_avg=st.global_avg, global_std=st.global_std)
        return out

    def batch_stats(self) -> dict:
        st = BatchStats()
        _check(lib().rf_batch_last_stats(self._h, C.byref(st)))
        return st.as_dict()

    def last_times(self):
        """(tables_ms, contract_ms, post_ms, kernel_launches) of the last call."""
        a, b, p = C.c_double(), C.c_double(), C.c_double()
        n = C.c_int32()
        _check(lib().rf_context_last_times(self._h, C.byref(a), C.byref(b), C.byref(p), C.byref(n)))
        return a.value, b.value, p.value, n.value
