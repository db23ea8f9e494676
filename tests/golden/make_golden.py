#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own format builders, COO CPU MTTKRP and CPU TTM (built as
oracle/_ref/libmmcsf_ref.so by oracle/build_ref.py from the reference's
sources; the MM-CSF builder also as oracle/_ref/libmmcsf_ref_heur.so, without
the partition override) on the reference's toy.tns and on seeded synthetic
tensors, and writes inputs and outputs as JSON. The tests compare both the C oracle and
the CUDA library against these files, so they run without the reference.

Usage: python tests/golden/make_golden.py [--reference <reference checkout>]
(default: $MMCSF_REFERENCE, else a `reference` directory beside this repository)
"""
import argparse
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import build_ref  # noqa: E402
from oracle import oracle as O  # noqa: E402

R_GOLD = 8


def _tolist(a):
    a = np.asarray(a)
    if a.dtype.kind == "f":
        return [float(x) for x in a]
    return [int(x) for x in a]


def _rand_tensor(rng, dims, n, skew=False, dup=False, ints=False):
    if skew:
        inds = [np.minimum(rng.zipf(1.6, n) - 1, d - 1).astype(np.uint64) for d in dims]
    else:
        inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    if not dup:
        key = np.zeros(n, np.uint64)
        for m, d in enumerate(dims):
            key = key * np.uint64(d) + inds[m]
        _, first = np.unique(key, return_index=True)
        first = np.sort(first)
        inds = [i[first] for i in inds]
    k = len(inds[0])
    vals = (rng.integers(1, 51, k).astype(np.float32) if ints
            else (rng.random(k) + 0.25).astype(np.float32))
    return inds, vals


def make_case(name, dims, inds, vals, tmp, runs, seed):
    path = os.path.join(tmp, name + ".tns")
    O.write_tns(path, dims, inds, vals)
    dims2, inds2, vals2 = O.load_tns(path)
    case = {"name": name, "dims": [int(d) for d in dims], "inds": [_tolist(i) for i in inds2],
            "vals": _tolist(vals2), "formats": [], "mttkrp": []}
    for kind, mode, fth in runs:
        d = O.ref_dump(kind, path, mode, fth, os.path.join(tmp, "dump.txt"))
        case["formats"].append({"kind": kind, "mode": mode, "f": int(fth),
                                "arrays": {k: _tolist(v) for k, v in d.items()}})
    rng = np.random.default_rng(seed)
    U = [rng.random((d, R_GOLD)).astype(np.float32) for d in dims]
    case["factors"] = [[_tolist(row) for row in u] for u in U]
    for m in range(len(dims)):
        out = O.ref_mttkrp_coo(dims2, inds2, vals2, m, U)
        case["mttkrp"].append({"mode": m, "R": R_GOLD, "out": [_tolist(row) for row in out]})
    with open(os.path.join(HERE, name + ".json"), "w") as fh:
        json.dump(case, fh, separators=(",", ":"))
    return name


def ttm_factor(rows, R):
    """The leaf factor of the TTM fixtures: a fixed formula, so the tests
    rebuild it exactly without storing it."""
    i = np.arange(rows, dtype=np.int64)[:, None]
    r = np.arange(R, dtype=np.int64)[None, :]
    return (((i * 31 + r * 17) % 97).astype(np.float32) / np.float32(97.0) + np.float32(0.01)).astype(np.float32)


def make_ttm(tmp, names):
    """ttm.json: the reference's TTM_CPU (its ttm command, src/ttm.cu) on the
    small 3-D cases above, every mode, -f none / 2, leaf factor ttm_factor."""
    out = {"R": R_GOLD, "runs": []}
    for name in names:
        with open(os.path.join(HERE, name + ".json")) as fh:
            case = json.load(fh)
        dims = case["dims"]
        if len(dims) != 3 or len(case["vals"]) > 160:
            continue
        inds = [np.asarray(i, np.uint64) for i in case["inds"]]
        vals = np.asarray(case["vals"], np.float32)
        path = os.path.join(tmp, name + "_ttm.tns")
        O.write_tns(path, dims, inds, vals)
        for mode in range(3):
            leaf = O.order_modes(dims, mode)[2]
            u = ttm_factor(dims[leaf], R_GOLD)
            for f in (0, 2):
                y, nf = O.ref_ttm(path, mode, f, u, len(vals) + 2)
                out["runs"].append({"case": name, "mode": mode, "f": f, "Y": [_tolist(r) for r in y]})
    with open(os.path.join(HERE, "ttm.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))


def make_heuristic(tmp, names):
    """heuristic.json: the reference's MM-CSF builder with its partition
    heuristic deciding (the build of oracle/_ref/libmmcsf_ref_heur.so, which
    drops the `mode = 2;` override of src/util.h:2517), on the cases above,
    for (-h, -f) = (1, none), (1, 3), (2, 3). Inputs the reference would read out of
    bounds on (the oracle says which) are skipped."""
    out = {"runs": []}
    for name in names:
        with open(os.path.join(HERE, name + ".json")) as fh:
            case = json.load(fh)
        dims = case["dims"]
        if len(case["vals"]) > 1000:
            continue
        inds = [np.asarray(i, np.uint64) for i in case["inds"]]
        vals = np.asarray(case["vals"], np.float32)
        path = os.path.join(tmp, name + "_heur.tns")
        O.write_tns(path, dims, inds, vals)
        d2, i2, v2 = O.load_tns(path)
        for h, f in ((1, O.INF_TH), (1, 3), (2, 3)):
            try:
                O.build_mmcsf(d2, i2, v2, mode=0, fbr_th=f, partition="heuristic", fbth=h)
            except ValueError:
                continue
            d = O.ref_dump_heuristic(path, 0, f, h, os.path.join(tmp, "dump.txt"))
            out["runs"].append({"case": name, "mode": 0, "h": h, "f": int(f),
                                "arrays": {k: _tolist(v) for k, v in d.items()}})
    with open(os.path.join(HERE, "heuristic.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=build_ref.REFERENCE_ROOT)
    ap.add_argument("--ttm-only", action="store_true", help="write ttm.json from the existing cases only")
    ap.add_argument("--heuristic-only", action="store_true",
                    help="write heuristic.json from the existing cases only")
    a = ap.parse_args()
    build_ref.build(os.path.join(a.reference, "src"))
    if a.ttm_only or a.heuristic_only:
        with open(os.path.join(HERE, "manifest.json")) as fh:
            names = json.load(fh)["cases"]
        if a.ttm_only:
            make_ttm(tempfile.mkdtemp(), names)
        if a.heuristic_only:
            build_ref.build(os.path.join(a.reference, "src"), variant="heuristic")
            make_heuristic(tempfile.mkdtemp(), names)
        return
    tmp = tempfile.mkdtemp()
    names = []
    INF = O.INF_TH
    # the reference's own fixture
    dims, inds, vals = O.load_tns(os.path.join(a.reference, "toy.tns"))
    runs = [(k, m, f) for k in ("mmcsf", "bcsf", "hyb") for m in range(3) for f in (1, 2, 128)]
    names.append(make_case("toy", dims, inds, vals, tmp, runs, seed=0))

    rng = np.random.default_rng(20261203)
    specs = [
        ("uni3d", [30, 25, 20], 400, dict()),
        ("skew3d", [40, 60, 25], 600, dict(skew=True)),
        ("dup3d", [6, 5, 7], 150, dict(dup=True)),
        ("equal3d", [12, 12, 12], 300, dict()),
        ("uni4d", [15, 9, 11, 5], 500, dict(ints=True)),
        ("skew4d", [50, 20, 10, 4], 900, dict(skew=True, ints=True)),
        ("fbrs4d", [3, 2, 4, 60], 700, dict()),
        ("single3d", [4, 4, 4], 1, dict()),
        ("single4d", [3, 3, 3, 3], 1, dict()),
    ]
    for name, dims, n, kw in specs:
        inds, vals = _rand_tensor(rng, dims, n, **kw)
        nd = len(dims)
        runs = []
        for kind in ("mmcsf", "bcsf", "hyb"):
            for f in (1, 3, INF):
                runs.append((kind, int(rng.integers(0, nd)), f))
        names.append(make_case(name, dims, inds, vals, tmp, runs, seed=len(names)))
    make_ttm(tmp, names)
    build_ref.build(os.path.join(a.reference, "src"), variant="heuristic")
    make_heuristic(tmp, names)
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump({"cases": names, "R": R_GOLD,
                   "source": "reference host code built by oracle/build_ref.py"}, fh, indent=1)
    print("wrote", names)


if __name__ == "__main__":
    main()
