#!/usr/bin/env python3
"""Build recipe for the reference-as-oracle library (test infrastructure).

Compiles isratnisa/MM-CSF's own host code (format builders in src/util.h, the
COO CPU MTTKRP in src/mttkrp_cpu.cpp and the CPU TTM in src/ttm_cpu.cpp)
together with oracle/ref_harness.cpp
into oracle/_ref/libmmcsf_ref.so.

The reference does not build as shipped with this image's g++ 13:
  * it includes Boost.Sort / Boost.Functional, which are not installed; the
    minimal stand-ins under oracle/shim/ replace them (sample_sort becomes a
    stable sort, so ties keep their prior order and results are deterministic);
  * dozens of `int` functions fall off their end without `return`, which g++
    13 compiles into traps or garbage. The recipe compiles with -Wreturn-type,
    and for every site the compiler reports it inserts `return 0;` before the
    closing brace.
Both edits are applied to a scratch copy under a temporary directory; the
reference tree is only read, nothing from it is written into this repository,
and the only outputs are the files under oracle/_ref/.

A second library, oracle/_ref/libmmcsf_ref_heur.so, is the same build with
one more edit: the unconditional `mode = 2;` that closes the nonzero loop of
mm_partition_reuseBased (src/util.h:2517) is removed, so the partition
heuristic above it decides. It pins the oracle's restatement of that
heuristic (run on one OpenMP thread: the loop decrements shared counters).

Usage: python oracle/build_ref.py [--src DIR] [--force]
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT_LIB = os.path.join(OUT_DIR, "libmmcsf_ref.so")
OUT_LIB_HEUR = os.path.join(OUT_DIR, "libmmcsf_ref_heur.so")
OUT_LIB_GPU = os.path.join(OUT_DIR, "libmmcsf_ref_gpu.so")
GPU_FILES = ["util.h", "mttkrp_gpu.h", "mttkrp_gpu.cu"]
NVCC_WARN_RE = re.compile(r"^(?P<file>[^(\s]+)\((?P<line>\d+)\): warning #940-D: missing return statement")
NVCCFLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++14", "-Xcompiler", "-fPIC,-fopenmp"]
OVERRIDE_RE = re.compile(r"^(\s*)mode = 2;\s*$")
# The reference checkout: $MMCSF_REFERENCE (its root) when set, else a
# directory named `reference` beside this repository.
REFERENCE_ROOT = os.environ.get("MMCSF_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
DEFAULT_SRC = os.path.join(REFERENCE_ROOT, "src")
FILES = ["util.h", "mttkrp_cpu.h", "mttkrp_cpu.cpp", "ttm_cpu.h", "ttm_cpu.cpp"]
CXXFLAGS = ["-std=c++14", "-fopenmp", "-fPIC", "-Wreturn-type"]
WARN_RE = re.compile(r"^(?P<file>[^:\s]+):(?P<line>\d+):(?P<col>\d+): warning: "
                     r"(no return statement in function returning non-void|"
                     r"control reaches end of non-void function)")


def _compile(build, src, obj, opt="-O3"):
    cmd = ["g++", opt] + CXXFLAGS + ["-I", build, "-I", os.path.join(HERE, "shim"), "-c", src, "-o", obj]
    p = subprocess.run(cmd, cwd=build, capture_output=True, text=True)
    return p


def _patch_missing_returns(build, stderr):
    sites = {}
    for line in stderr.splitlines():
        m = WARN_RE.match(line)
        if not m:
            continue
        fname = os.path.basename(m.group("file"))
        sites.setdefault(fname, set()).add((int(m.group("line")), int(m.group("col"))))
    n = 0
    for fname, locs in sites.items():
        path = os.path.join(build, fname)
        if not os.path.exists(path):
            continue
        with open(path) as fh:
            lines = fh.readlines()
        for ln, col in sorted(locs, reverse=True):
            # The report points at the closing brace, or (for "control reaches
            # end") at the last statement; patch the first '}' from there on.
            li, c = ln - 1, col - 1
            while li < len(lines):
                j = lines[li].find("}", c)
                if j >= 0:
                    lines[li] = lines[li][:j] + "return 0; " + lines[li][j:]
                    n += 1
                    break
                li, c = li + 1, 0
        with open(path, "w") as fh:
            fh.writelines(lines)
    return n


def _patch_nvcc_missing_returns(build, stderr):
    """The same `return 0;` patch for the sites nvcc reports (warning #940,
    at the function's closing brace)."""
    sites = {}
    for line in stderr.splitlines():
        m = NVCC_WARN_RE.match(line)
        if m:
            sites.setdefault(os.path.basename(m.group("file")), set()).add(int(m.group("line")))
    n = 0
    for fname, lns in sites.items():
        path = os.path.join(build, fname)
        if not os.path.exists(path):
            continue
        with open(path) as fh:
            lines = fh.readlines()
        for ln in sorted(lns, reverse=True):
            li = ln - 1
            while li < len(lines):
                j = lines[li].find("}")
                if j >= 0:
                    lines[li] = lines[li][:j] + "return 0; " + lines[li][j:]
                    n += 1
                    break
                li += 1
        with open(path, "w") as fh:
            fh.writelines(lines)
    return n


def build_gpu(src=DEFAULT_SRC, force=False, verbose=True):
    """The reference's GPU MTTKRP (src/mttkrp_gpu.cu, all of its kernels and
    drivers) compiled for sm_100a with nvcc, plus oracle/ref_gpu_harness.cu,
    into oracle/_ref/libmmcsf_ref_gpu.so, from a scratch copy with the same
    missing-return patch."""
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found at {src}")
    if os.path.exists(OUT_LIB_GPU) and not force:
        return OUT_LIB_GPU
    os.makedirs(OUT_DIR, exist_ok=True)
    build_dir = tempfile.mkdtemp(prefix="mmcsf_ref_gpu_build_")
    try:
        for f in GPU_FILES:
            shutil.copy(os.path.join(src, f), os.path.join(build_dir, f))
            os.chmod(os.path.join(build_dir, f), 0o644)
        units = [(os.path.join(build_dir, "mttkrp_gpu.cu"), os.path.join(build_dir, "mttkrp_gpu.o")),
                 (os.path.join(HERE, "ref_gpu_harness.cu"), os.path.join(build_dir, "harness.o"))]
        total = 0
        for _ in range(4):
            patched = 0
            for srcf, obj in units:
                cmd = ["nvcc"] + NVCCFLAGS + ["-I", build_dir, "-I", os.path.join(HERE, "shim"), "-c", srcf, "-o", obj]
                p = subprocess.run(cmd, cwd=build_dir, capture_output=True, text=True)
                if p.returncode != 0:
                    raise RuntimeError(f"compiling {srcf} failed:\n{p.stderr[-4000:]}")
                patched += _patch_nvcc_missing_returns(build_dir, p.stderr)
            total += patched
            if patched == 0:
                break
        else:
            raise RuntimeError("missing-return patching did not converge")
        cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fopenmp", "-o",
               OUT_LIB_GPU] + [o for _, o in units] + ["-lgomp"]
        subprocess.run(cmd, check=True, cwd=build_dir)
        if verbose:
            print(f"built {OUT_LIB_GPU} ({total} missing-return sites patched in the scratch copy)")
        return OUT_LIB_GPU
    finally:
        shutil.rmtree(build_dir, ignore_errors=True)


def _remove_partition_override(build):
    """Drop the `mode = 2;` directly above the `/*populate new partitions*/`
    comment in mm_partition_reuseBased (src/util.h:2517)."""
    path = os.path.join(build, "util.h")
    with open(path) as fh:
        lines = fh.readlines()
    start = next(i for i, l in enumerate(lines) if "inline int mm_partition_reuseBased(" in l)
    end = next(i for i in range(start + 1, len(lines)) if lines[i].startswith("inline ") or
               lines[i].startswith("// more detailed check"))
    sites = []
    for i in range(start, end):
        if OVERRIDE_RE.match(lines[i]):
            nxt = next((j for j in range(i + 1, end) if lines[j].strip()), None)
            if nxt is not None and "populate new partitions" in lines[nxt]:
                sites.append(i)
    if len(sites) != 1:
        raise RuntimeError(f"expected one partition override in mm_partition_reuseBased, found {len(sites)}")
    i = sites[0]
    lines[i] = OVERRIDE_RE.sub(r"\1/* override removed */", lines[i]) + "\n"
    with open(path, "w") as fh:
        fh.writelines(lines)
    return i + 1


def build(src=DEFAULT_SRC, force=False, verbose=True, variant="shipped"):
    """variant "shipped": the reference as it is (libmmcsf_ref.so);
    "heuristic": without the partition override (libmmcsf_ref_heur.so)."""
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found at {src}")
    out_lib = OUT_LIB if variant == "shipped" else OUT_LIB_HEUR
    if os.path.exists(out_lib) and not force:
        return out_lib
    os.makedirs(OUT_DIR, exist_ok=True)
    build_dir = tempfile.mkdtemp(prefix="mmcsf_ref_build_")
    try:
        for f in FILES:
            shutil.copy(os.path.join(src, f), os.path.join(build_dir, f))
            os.chmod(os.path.join(build_dir, f), 0o644)
        if variant == "heuristic":
            ln = _remove_partition_override(build_dir)
            if verbose:
                print(f"removed the partition override at util.h:{ln} in the scratch copy")
        harness = os.path.join(HERE, "ref_harness.cpp")
        units = [(harness, os.path.join(build_dir, "harness.o")),
                 (os.path.join(build_dir, "mttkrp_cpu.cpp"), os.path.join(build_dir, "mttkrp_cpu.o")),
                 (os.path.join(build_dir, "ttm_cpu.cpp"), os.path.join(build_dir, "ttm_cpu.o"))]
        total = 0
        for _ in range(8):
            patched = 0
            # -O0 and -O3 report different subsets of the sites; patch both.
            for opt in ("-O0", "-O3"):
                for srcf, obj in units:
                    p = _compile(build_dir, srcf, obj, opt)
                    if p.returncode != 0:
                        raise RuntimeError(f"compiling {srcf} failed:\n{p.stderr[-4000:]}")
                    patched += _patch_missing_returns(build_dir, p.stderr)
            total += patched
            if patched == 0:
                break
        else:
            raise RuntimeError("missing-return patching did not converge")
        cmd = ["g++", "-shared", "-fopenmp", "-o", out_lib] + [o for _, o in units]
        subprocess.run(cmd, check=True, cwd=build_dir)
        if verbose:
            print(f"built {out_lib} ({total} missing-return sites patched in the scratch copy)")
        return out_lib
    finally:
        shutil.rmtree(build_dir, ignore_errors=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(a.src, a.force)
        build(a.src, a.force, variant="heuristic")
        build_gpu(a.src, a.force)
    except Exception as e:  # noqa: BLE001
        print(f"reference build failed: {e}", file=sys.stderr)
        sys.exit(1)
