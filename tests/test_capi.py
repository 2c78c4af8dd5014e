"""C-ABI host logic, no GPU needed: the library loads and exports every
symbol include/randomfield_b200.h declares, option defaults, the reference's
validation rules as status codes (type_inputRF.f90:1159-1206,
randomFieldND.f90:162-166), the wavevector geometry against the oracle, and
a loud failure (no CPU fallback) when no GPU is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.helpers import grid, uniform_points

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "randomfield_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rf_[a-z_0-9]+)\s*\(", text)))


def test_header_and_exports_agree():
    syms = declared_symbols()
    assert set(syms) == set(rf.EXPORTS)
    L = rf.lib()
    for s in syms:
        assert hasattr(L, s), s


def test_fortran_module_binds_exported_symbols():
    """Every bind(C) name of the Fortran module (except libc's strlen) is a
    symbol the header declares and the library exports."""
    f90 = os.path.join(os.path.dirname(HEADER), "..", "randomfield_b200", "fortran", "rf_gpu.f90")
    names = set(re.findall(r'bind\(C,\s*name="([a-z_0-9]+)"\)', open(f90).read())) - {"strlen"}
    assert "rf_create_standard_gaussian_field_grid" in names
    assert names <= set(declared_symbols())
    L = rf.lib()
    for s in names:
        assert hasattr(L, s), s


def test_abi_version_and_option_defaults():
    assert rf.lib().rf_abi_version() == 1
    o = rf.Options()
    rf.lib().rf_options_init(C.byref(o))
    assert o.size == C.sizeof(rf.Options)  # the C and ctypes layouts agree
    assert o.precision == rf.PREC_BF16 and o.seed_start == 0 and o.device == 0
    assert list(o.k_nstep) == [0, 0, 0] and o.literal == 0 and o.normalize == 0


def call(x, nDim=3, n=None, corrMod=1, margiFirst=1, corrL=(1.0, 1.0, 1.0), fieldAvg=0.0, fieldVar=1.0, Nmc=2,
         method=2, out=True, opts=None):
    L = rf.lib()
    x = np.asfortranarray(np.asarray(x, dtype=np.float64))
    n = x.shape[1] if n is None else n
    cl = np.asarray(corrL, dtype=np.float64)
    res = np.zeros((max(n, 1), max(Nmc, 1)), order="F") if out else None
    P = C.POINTER(C.c_double)
    o = opts or rf.Options.make()
    rc = L.rf_create_standard_gaussian_field_unstruct(
        x.ctypes.data_as(P), nDim, n, corrMod, margiFirst, cl.ctypes.data_as(P), fieldAvg, fieldVar, Nmc, method,
        res.ctypes.data_as(P) if out else None, C.byref(o))
    return rc, L.rf_last_error().decode()


@pytest.mark.parametrize("kw,code", [
    (dict(Nmc=0), -1),
    (dict(nDim=4), -2),
    (dict(corrL=(1.0, 0.0, 1.0)), -3),
    (dict(corrL=(1.0, 1.0, -2.0)), -3),
    (dict(margiFirst=2, fieldAvg=0.0), -4),
    (dict(margiFirst=2, fieldAvg=-1.0), -4),
    (dict(method=4), -5),
    (dict(method=0), -5),
    (dict(method=1, opts=rf.Options.make(literal=True)), -9),
    (dict(corrMod=3), -6),
    (dict(margiFirst=0), -7),
    (dict(out=False), -9),
    (dict(n=0), -9),
    (dict(opts=rf.Options.make(precision=7)), -9),
    (dict(opts=rf.Options.make(k_nstep=(1, 4, 4))), -9),
    (dict(method=2, opts=rf.Options.make(literal=True), margiFirst=1), None),
])
def test_validation_codes(kw, code):
    x = grid(4, 0.5).T
    rc, msg = call(x, **kw)
    if code is None:
        return  # valid request: needs a GPU, covered in the GPU suite
    assert rc == code, (rc, msg)
    assert msg


def test_isotropic_needs_2d_or_3d():
    x = np.linspace(0, 1, 10).reshape(1, -1)
    rc, msg = call(x, nDim=1, method=1, corrL=(1.0,))
    assert rc == -2 and "isotropic" in msg


def test_python_mirror_errors():
    x = grid(4, 0.5).T
    with pytest.raises(rf.RandomFieldError) as e:
        rf.create_standard_gaussian_field_unstruct(x, "gaussian", "lognormal", [1, 1, 1], 0.0, 1.0, 2, 2)
    assert e.value.code == -4 and e.value.status == "RF_EINVAL_LOGNORMAL"
    with pytest.raises(rf.RandomFieldError) as e:
        rf.create_standard_gaussian_field_unstruct(x, "exponential", "gaussian", [1, 1, 1], 0.0, 1.0, 2, 2)
    assert e.value.code == -9
    with pytest.raises(rf.RandomFieldError):
        rf.create_standard_gaussian_field_unstruct(x, "gaussian", "gaussian", [1, 1, 1], 0.0, 1.0, 2, 2,
                                                   randField=np.zeros((64, 2)))  # C order


@pytest.mark.parametrize("case", [
    dict(pts="grid32", method=2),
    dict(pts="grid32", method=2, kNStep=(16, 16, 16)),
    dict(pts="uniform", method=2, corrL=(2.0, 1.0, 0.5)),
    dict(pts="uniform", method=1),
    dict(pts="uniform", method=1, isoNRadial=64, isoNDir=64),
    dict(pts="uniform2d", method=2, corrL=(0.7, 1.3)),
])
def test_geometry_matches_oracle(case):
    pts = {"grid32": grid(32, 0.1), "uniform": uniform_points(2000, 10.0),
           "uniform2d": uniform_points(500, 5.0, nDim=2)}[case["pts"]]
    nDim = pts.shape[1]
    corrL = case.get("corrL", (1.0,) * nDim)
    kn = case.get("kNStep", (0, 0, 0))
    g = O.OracleRequest(pts, method=case["method"], corrL=corrL, kNStep=kn, isoNRadial=case.get("isoNRadial", 0),
                        isoNDir=case.get("isoNDir", 0)).geometry()
    K, kNStep, kDelta, amp = rf.query_geometry(pts.T, "gaussian", corrL, case["method"], k_nstep=kn,
                                               iso_n_radial=case.get("isoNRadial", 0),
                                               iso_n_dir=case.get("isoNDir", 0))
    assert K == g.K
    assert kNStep[:2] == list(g.kNStep)[:2]
    assert kDelta[0] == g.kDelta[0]
    assert amp == g.ampMult


def test_zero_extent_is_rejected():
    x = np.zeros((3, 5))
    with pytest.raises(rf.RandomFieldError) as e:
        rf.query_geometry(x, "gaussian", [1, 1, 1], 2)
    assert e.value.code == -8
    # an explicit extent makes a single point valid
    K, *_ = rf.query_geometry(x, "gaussian", [1, 1, 1], 2, x_range=(1.0, 1.0, 1.0))
    assert K > 0


def test_no_gpu_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    x = grid(4, 0.5).T
    rc, msg = call(x)
    assert rc == -25 and "device" in msg
    with pytest.raises(rf.RandomFieldError) as e:
        rf.create_standard_gaussian_field_grid((0.0, 0.0, 0.0), (0.5, 0.5, 0.5), (4, 4, 4), 1, 1, (1.0, 1.0, 1.0),
                                               0.0, 1.0, 2)
    assert e.value.code == -25


def test_grid_entry_validates_before_touching_a_device():
    """The structured-grid entry point's argument checks are host-side."""
    base = dict(xMin=(0.0, 0.0, 0.0), xStep=(0.1, 0.1, 0.1), xNStep=(8, 8, 8), corrMod=1, margiFirst=1,
                corrL=(1.0, 1.0, 1.0), fieldAvg=0.0, fieldVar=1.0, Nmc=2)
    for kw, code in ((dict(Nmc=0), -1), (dict(corrL=(1.0, -1.0, 1.0)), -3), (dict(method=5), -5),
                     (dict(method=1), -10), (dict(xStep=(0.1, 0.0, 0.1)), -9), (dict(k_nstep=(33, 4, 4)), -10),
                     (dict(margiFirst=2, fieldAvg=-1.0), -4)):
        a = dict(base)
        opts = {k: kw.pop(k) for k in list(kw) if k in ("k_nstep",)}
        a.update(kw)
        with pytest.raises(rf.RandomFieldError) as e:
            rf.create_standard_gaussian_field_grid(**a, **opts)
        assert e.value.code == code, kw


def test_blend_layout_rounds_overlap_and_checks_the_split():
    """rf_blend_layout (host only): topography_RF.f90:49-52 overlap rounding
    and localization_RF.f90:746 overlapNPoints; subdomains share O points."""
    g = rf.BlendGrid.make((21, 21, 21), (0.1, 0.1, 0.1), (2, 2, 2), 0.4)
    assert rf.blend_layout(g, (1.0, 1.0, 1.0)) == ([12, 12, 12], [3, 3, 3])
    # overlap below two steps on a split axis is raised to two steps: O = 1
    g = rf.BlendGrid.make((21, 21), (0.1, 0.1), (2, 1), 0.05)
    L, O = rf.blend_layout(g, (1.0, 1.0))
    assert O[0] == 1 and L[0] == 11 and L[1] == 21 and O[1] < 1
    g = rf.BlendGrid.make((256, 256, 256), (0.05,) * 3, (2, 2, 2), 0.65)
    assert rf.blend_layout(g, (1.0, 1.0, 1.0)) == ([134, 134, 134], [12, 12, 12])
    g = rf.BlendGrid.make((20, 20, 20), (0.1,) * 3, (2, 2, 2), 0.4)
    with pytest.raises(rf.RandomFieldError) as e:
        rf.blend_layout(g, (1.0, 1.0, 1.0))
    assert e.value.code == -8
