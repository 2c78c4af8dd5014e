"""Builds tests/sanitize/_build/capi_harness: every source of the library
compiled with the host code under AddressSanitizer and UBSan (device code as
the library builds it), linked with capi_harness.cpp.  Incremental; used by
tests/test_sanitizers.py."""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BUILD = os.path.join(HERE, "_build")
CSRC = os.path.join(ROOT, "randomfield_b200", "csrc")
INC = os.path.join(ROOT, "include")
EXE = os.path.join(BUILD, "capi_harness")
SAN = ["-Xcompiler", "-fsanitize=address", "-Xcompiler", "-fsanitize=undefined", "-Xcompiler",
       "-fno-sanitize-recover=undefined", "-Xcompiler", "-fno-omit-frame-pointer"]


def _nvcc():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from randomfield_b200 import build as b

    return b.NVCC, b.ARCH, b.SOURCES


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(d) > os.path.getmtime(target) for d in deps)


def build() -> str:
    nvcc, arch, sources = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(INC, "randomfield_b200.h"))

    def one(src):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _stale(obj, [src] + hdrs):
            cmd = [nvcc, *arch, "-O1", "-g", "-std=c++17", "--expt-relaxed-constexpr", "-I", INC, *SAN, "-c", src,
                   "-o", obj]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        return obj

    srcs = [os.path.join(CSRC, s) for s in sources] + [os.path.join(HERE, "capi_harness.cpp")]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(one, srcs))
    if _stale(EXE, objs):
        r = subprocess.run([nvcc, *arch, *SAN, "-o", EXE, *objs, "-lpthread"], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return EXE


if __name__ == "__main__":
    print(build())
