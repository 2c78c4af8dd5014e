"""The RF_DEBUG_BOUNDS build (librf_b200_bounds.so): device index checks that
record a failed check in the context's error word and skip the access, the
stand-in for a device memory checker (compute-sanitizer is closed on the
GPU pool).

Run in a child process with RF_LIB pointing at the checked library:
  - its self test plants an index one past a buffer; the check catches it,
    the call reports RF_EBOUNDS, and the context then generates a field
    identical to a fresh context's;
  - generations through every kernel family (outer-group contraction, the
    tcgen05 contraction with the FP8 form, the plain FP32 form, the table
    generator, a grouped batch, a blend on the structured-grid path) report
    no failed check and give the normal library's fields bit for bit.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import randomfield_b200 as rf

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BOUNDS_LIB = os.path.join(ROOT, "randomfield_b200", "librf_b200_bounds.so")

WORKLOADS = r'''
import sys, numpy as np
sys.path.insert(0, ROOT)
import randomfield_b200 as rf
from tests.helpers import grid, uniform_points

def fields():
    out = {}
    g = grid(18, 0.1)
    iso = uniform_points(4000, 6.0, seed=3)
    for prec in ("bf16", "fp8", "fp32"):
        out["grid_" + prec] = np.asarray(rf.create_standard_gaussian_field_unstruct(
            g.T, "gaussian", "lognormal", [1.0, 0.7, 1.3], 1.0, 0.25, 6, rf.SHINOZUKA, precision=prec,
            k_nstep=(10, 12, 9), seed_start=4))
    out["iso_bf16"] = np.asarray(rf.create_standard_gaussian_field_unstruct(
        iso.T, "gaussian", "gaussian", [1.0] * 3, 0.0, 1.0, 5, rf.ISOTROPIC, precision="bf16", iso_n_radial=16,
        iso_n_dir=12, seed_start=2))
    ctx = rf.Context(0)
    reqs, outs = [], []
    for i, (pts, meth, o) in enumerate([(g, rf.SHINOZUKA, dict(k_nstep=(24, 24, 24))),
                                         (iso, rf.ISOTROPIC, dict(iso_n_radial=16, iso_n_dir=12)),
                                         (g[:1000], rf.SHINOZUKA, dict(k_nstep=(24, 24, 24)))]):
        xa = np.asfortranarray(pts.T)
        oa = np.empty((pts.shape[0], 3 + i), order="F")
        outs.append((xa, oa))
        reqs.append(rf.make_request(xa, "gaussian", "gaussian", [1.0] * 3, 0.0, 1.0, 3 + i, meth, oa,
                                    precision="bf16", seed_start=10 + i, **o))
    rf.generate_batch(ctx, reqs)
    for i, (_, oa) in enumerate(outs):
        out["batch_%d" % i] = oa.copy()
    bg = rf.BlendGrid.make((21, 21, 21), (0.1, 0.1, 0.1), (2, 2, 2), 0.4)
    out["blend"] = ctx.generate_blended(bg, "gaussian", "gaussian", (1.0, 1.0, 1.0), 0.0, 1.0, 2, 2,
                                        precision="bf16", seed_start=5, k_nstep=(12, 12, 12))
    ctx.close()
    return out
'''

CHILD = WORKLOADS + r'''
assert rf.lib().rf_debug_bounds_build() == 1
ctx = rf.Context(0)
try:
    ctx.selftest_bounds()
    raise SystemExit("the planted index was not caught")
except rf.RandomFieldError as e:
    assert e.code == -26, e
g = grid(12, 0.1)
a = np.zeros((g.shape[0], 3), order="F")
import torch
dx = torch.from_numpy(np.ascontiguousarray(g)).cuda()
d1 = torch.empty((3, g.shape[0]), dtype=torch.float64, device="cuda")
d2 = torch.empty_like(d1)
ctx.generate(dx, 3, g.shape[0], 1, 1, [1.0] * 3, 0.0, 1.0, 3, rf.SHINOZUKA, d1, k_nstep=(8, 8, 8))
ctx.synchronize()
c2 = rf.Context(0)
c2.generate(dx, 3, g.shape[0], 1, 1, [1.0] * 3, 0.0, 1.0, 3, rf.SHINOZUKA, d2, k_nstep=(8, 8, 8))
c2.synchronize()
assert torch.equal(d1, d2)
ctx.close(); c2.close()
np.savez(OUT, **fields())
print("child ok")
'''


def test_bounds_build_checks_and_matches_the_normal_build():
    if not os.path.exists(BOUNDS_LIB):
        pytest.fail(f"{BOUNDS_LIB} is missing: run `python -m randomfield_b200.build --debug-bounds`")
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "bounds.npz")
        env = dict(os.environ, RF_LIB=BOUNDS_LIB)
        code = f"ROOT = {ROOT!r}\nOUT = {out!r}\n" + CHILD
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0 and "child ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
        checked = dict(np.load(out))
    assert rf.lib().rf_debug_bounds_build() == 0
    ns = {"ROOT": ROOT}
    exec(compile(WORKLOADS, "workloads", "exec"), ns)
    normal = ns["fields"]()
    assert set(normal) == set(checked)
    for k in normal:
        assert np.isfinite(normal[k]).all(), k
        assert np.array_equal(np.asarray(normal[k]), checked[k]), k
