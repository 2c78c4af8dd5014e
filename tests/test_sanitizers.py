"""Host code under AddressSanitizer and UBSan (no GPU involved).

- The C oracle (the checker of every parity test): `make -C oracle sanitize`
  builds it with -fsanitize=address,undefined; tests/sanitize/
  exercise_oracle.py drives every entry point (rnglib, the four methods,
  literal mode, cm_COS, lognormal and normalisation, row subsets on two
  threads, the recast and baseline loops, marginal, grid and partition
  helpers) in a child process with libasan preloaded.
- The C-ABI's host paths: tests/sanitize/build_harness.py compiles every
  library source with the host code instrumented and links
  tests/sanitize/capi_harness.cpp, which runs the validation codes, the
  geometry, the blend layout, the structured-grid refusals and the result
  writer.
Any sanitizer report fails the test (UBSan halts on the first error).
"""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = os.path.join(ROOT, "tests", "sanitize")


def _libasan():
    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    p = subprocess.run([gcc, "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    if not p or not os.path.isabs(p) or not os.path.exists(p):
        pytest.skip("no libasan for the host compiler")
    return p


def _env(**kw):
    env = dict(os.environ)
    env.update(ASAN_OPTIONS="detect_leaks=0:protect_shadow_gap=0", UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    env.update(kw)
    return env


def _clean(out):
    assert "AddressSanitizer" not in out and "runtime error" not in out, out[-4000:]


def test_oracle_under_asan_and_ubsan():
    asan = _libasan()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "sanitize"], check=True)
    lib = os.path.join(ROOT, "oracle", "_san", "librfo.so")
    r = subprocess.run([sys.executable, os.path.join(SAN, "exercise_oracle.py")], capture_output=True, text=True,
                       env=_env(LD_PRELOAD=asan, RFO_LIB=lib), timeout=600)
    _clean(r.stdout + r.stderr)
    assert r.returncode == 0 and "exercised" in r.stdout, (r.stdout + r.stderr)[-4000:]


def test_capi_host_paths_under_asan_and_ubsan(tmp_path):
    _libasan()
    sys.path.insert(0, SAN)
    try:
        import build_harness
    finally:
        sys.path.remove(SAN)
    exe = build_harness.build()
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, env=_env(), timeout=600)
    _clean(r.stdout + r.stderr)
    assert r.returncode == 0 and "harness ok" in r.stdout, (r.stdout + r.stderr)[-4000:]
    assert (tmp_path / "h5" / "h3.h5").exists() and (tmp_path / "xmf" / "h3.xmf").exists()
