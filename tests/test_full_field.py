"""Whole-field parity at the headline size (128^3 grid, 24^3 x 4
wavevectors, Nmc 64): every value of the device field against an FP64
reference of the same field.

The reference is tests/helpers.py::separable_field: the oracle's own
wavevectors and phases (rfo_phase_matrix) summed axis by axis with complex
matrix products, which turns the 1.2e11 cosines of the point-by-point sum
into seconds of BLAS.  It is pinned here on the CPU against the oracle's
point-by-point sum (rfo_generate) on rows of the same 128^3 workload and on
small grids in 1-D to 3-D; the GPU tests then compare all 134 M values of the
BF16 and FP16 forms (relative-L2 <= 2e-3 overall and for every
realization; the BF16 form, the outer-group contraction with its TF32 K-steps,
also within 1.5e-3 for every realization, its margin under the bound) and of
the structured-grid path (<= 1e-11).
"""
import numpy as np
import pytest

import randomfield_b200 as rf
from oracle import oracle as O
from tests.helpers import grid, separable_field

HEAD = dict(xMin=(0.0, 0.0, 0.0), xStep=(0.05, 0.05, 0.05), xNStep=(128, 128, 128), corrL=(2.0, 1.0, 0.5),
            kNStep=(24, 24, 24))


@pytest.mark.parametrize("nd", [1, 2, 3])
def test_separable_reference_small_grids(nd):
    xMin, xStep, xNStep = (0.3, -1.0, 2.0)[:nd], (0.21, 0.17, 0.3)[:nd], (9, 7, 5)[:nd]
    corrL = (1.0, 2.0, 0.5)[:nd]
    for kn, cm in (((6, 5, 4)[:nd], O.CM_GAUSSIAN), ((0, 0, 0)[:nd], O.CM_GAUSSIAN), ((8, 4, 3)[:nd], O.CM_COS)):
        ref = O.OracleRequest(O.grid(xMin, xStep, xNStep), corrL=corrL, Nmc=3, kNStep=kn, seedStart=2,
                              corrMod=cm).generate()
        f = separable_field(xMin, xStep, xNStep, corrL, 3, kNStep=kn, seedStart=2, corrMod=cm)
        np.testing.assert_allclose(f, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_separable_reference_on_the_headline_workload():
    x = grid(128, 0.05)
    rows = np.random.RandomState(4).choice(x.shape[0], 64, replace=False)
    ref = O.OracleRequest(x, corrL=HEAD["corrL"], Nmc=2, kNStep=HEAD["kNStep"]).generate(rows=rows)
    f = separable_field(HEAD["xMin"], HEAD["xStep"], HEAD["xNStep"], HEAD["corrL"], 2, kNStep=HEAD["kNStep"])
    assert np.abs(f[:, rows] - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.fixture(scope="module")
def head_ref():
    return separable_field(HEAD["xMin"], HEAD["xStep"], HEAD["xNStep"], HEAD["corrL"], 64, kNStep=HEAD["kNStep"])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_whole_field_tensor_core_forms(head_ref, prec):
    x = grid(128, 0.05)
    out = rf.create_standard_gaussian_field_unstruct(x.T, "gaussian", "gaussian", HEAD["corrL"], 0.0, 1.0, 64,
                                                     rf.SHINOZUKA, precision=prec, k_nstep=HEAD["kNStep"])
    got = np.asarray(out).T
    d = got - head_ref
    assert np.linalg.norm(d) <= 2e-3 * np.linalg.norm(head_ref)
    per = np.linalg.norm(d, axis=1) / np.linalg.norm(head_ref, axis=1)
    assert per.max() <= 2e-3, per.max()
    if prec == "bf16":
        assert per.max() <= 1.5e-3, per.max()


@pytest.mark.gpu
def test_whole_field_structured_grid_path(head_ref):
    out = rf.create_standard_gaussian_field_grid(HEAD["xMin"], HEAD["xStep"], HEAD["xNStep"], "gaussian",
                                                 "gaussian", HEAD["corrL"], 0.0, 1.0, 64, k_nstep=HEAD["kNStep"])
    got = np.asarray(out).T
    assert np.linalg.norm(got - head_ref) <= 1e-11 * np.linalg.norm(head_ref)
