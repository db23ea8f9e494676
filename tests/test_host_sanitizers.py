"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU only).

Builds tests/sanitize/host_checks.cpp with the library's host COO MTTKRP
(mm-csf_b200/csrc/coo_host.cpp, status.cpp) and the oracle's C sources, all
with -fsanitize=address,undefined, and runs it: the seeded generator, the
sort, the CSF builder and both COO MTTKRPs on 3-D and 4-D tensors, with the
host MTTKRP checked against the oracle. Any sanitizer report fails the run.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_host_code_sanitizers(tmp_path):
    if not shutil.which("g++") or not shutil.which("gcc"):
        pytest.skip("no host compiler")
    if not os.path.isfile(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("no CUDA headers")
    san = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-g", "-O1"]
    objs = []
    for src in ("oracle/mmcsf_oracle.c", "oracle/generate.c"):
        obj = str(tmp_path / (os.path.basename(src) + ".o"))
        subprocess.run(["gcc", "-std=c11", "-D_GNU_SOURCE", *san, "-c", os.path.join(ROOT, src), "-o", obj],
                       check=True)
        objs.append(obj)
    exe = str(tmp_path / "host_checks")
    srcs = [os.path.join(ROOT, p) for p in ("tests/sanitize/host_checks.cpp", "mm-csf_b200/csrc/coo_host.cpp",
                                             "mm-csf_b200/csrc/status.cpp")]
    subprocess.run(["g++", "-std=c++17", *san, "-I", os.path.join(CUDA, "include"), *srcs, *objs,
                    "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-pthread", "-lm", "-o", exe], check=True)
    env = dict(os.environ, ASAN_OPTIONS="abort_on_error=0:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1",
               LD_LIBRARY_PATH=os.path.join(CUDA, "lib64") + ":" + os.environ.get("LD_LIBRARY_PATH", ""))
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "host checks passed" in r.stdout
