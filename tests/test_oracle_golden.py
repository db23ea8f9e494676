"""The oracle is pinned to the reference: every array the reference's own
builders produced (tests/golden/, made by tests/golden/make_golden.py from
the reference's sources) must come out of the C restatement unchanged."""
import numpy as np
import pytest

from oracle import oracle as O


def _inputs(case):
    dims = case["dims"]
    inds = [np.array(i, dtype=np.uint64) for i in case["inds"]]
    vals = np.array(case["vals"], dtype=np.float32)
    return dims, inds, vals


def test_format_arrays_match_reference(golden_cases):
    n = 0
    for case in golden_cases:
        dims, inds, vals = _inputs(case)
        for fmt in case["formats"]:
            build = {"mmcsf": O.build_mmcsf, "bcsf": O.build_bcsf, "hyb": O.build_hyb}[fmt["kind"]]
            got = build(dims, inds, vals, fmt["mode"], fmt["f"])
            for k, v in fmt["arrays"].items():
                assert k in got, (case["name"], fmt["kind"], k)
                want = np.array(v, dtype=got[k].dtype)
                assert np.array_equal(got[k], want), (case["name"], fmt["kind"], fmt["mode"], fmt["f"], k)
                n += 1
    assert n > 500


def test_coo_mttkrp_bit_exact_to_reference(golden_cases):
    for case in golden_cases:
        dims, inds, vals = _inputs(case)
        U = [np.array(u, dtype=np.float32).reshape(d, -1) for u, d in zip(case["factors"], dims)]
        for mt in case["mttkrp"]:
            got = O.mttkrp_coo_f32(inds, vals, mt["mode"], U)
            want = np.array(mt["out"], dtype=np.float32).reshape(got.shape)
            assert np.array_equal(got, want), (case["name"], mt["mode"])


def test_toy_known_answer():
    """toy.tns with the reference's constant factors U[m] = m + 0.5
    (src/util.h:3223): slice sums times the other two constants."""
    dims = [3, 3, 3]
    coords = [(1, 1, 1, 1.0), (1, 2, 2, 2.0), (1, 3, 1, 10.0), (2, 1, 3, 7.0), (2, 3, 1, 6.0),
              (2, 3, 2, 5.0), (3, 1, 3, 3.0), (3, 2, 2, 11.0)]
    inds = [np.array([c[m] - 1 for c in coords], np.uint64) for m in range(3)]
    vals = np.array([c[3] for c in coords], np.float32)
    U = [np.full((3, 4), m + 0.5, np.float32) for m in range(3)]
    # the reference's -t 1 output adds (mode + 0.5) because it never zeroes
    want = {0: [49.25, 68.00, 53.00], 1: [15.25, 17.75, 27.75], 2: [15.25, 16.00, 10.00]}
    for mode in range(3):
        got = O.mttkrp_coo_f32(inds, vals, mode, U)[:, 0] + (mode + 0.5)
        assert np.allclose(got, want[mode]), (mode, got)


def test_mode_order_rule():
    assert O.order_modes([1000, 1000, 1000], 2) == [2, 0, 1]
    assert O.order_modes([500000, 2000000, 20000], 2) == [2, 0, 1]
    assert O.order_modes([1000000, 20000, 5000, 200], 2) == [2, 3, 1, 0]
    assert O.order_modes([100000, 50000, 10000], 2) == [2, 1, 0]
    orders = [O.order_modes([1000] * 3, m) for m in range(3)]
    assert O.redundant_mode(orders) == 1


@pytest.mark.skipif(not O.ref_available(), reason="reference oracle not built here")
def test_reference_library_agrees_on_fresh_random_tensor(tmp_path):
    rng = np.random.default_rng(5)
    dims = [9, 14, 6, 5]
    n = 400
    inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    vals = (rng.random(n) + 0.1).astype(np.float32)
    p = str(tmp_path / "t.tns")
    O.write_tns(p, dims, inds, vals)
    dims2, inds2, vals2 = O.load_tns(p)
    for kind, build in (("mmcsf", O.build_mmcsf), ("bcsf", O.build_bcsf), ("hyb", O.build_hyb)):
        ref = O.ref_dump(kind, p, 1, 2, str(tmp_path / "d.txt"))
        got = build(dims2, inds2, vals2, 1, 2)
        for k, v in ref.items():
            assert np.array_equal(got[k], v.astype(got[k].dtype)), (kind, k)


def _heuristic_runs():
    import json
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with open(os.path.join(here, "heuristic.json")) as fh:
        return json.load(fh)["runs"]


def test_partition_heuristic_matches_reference(golden_cases):
    """The restated partition heuristic (mm_partition_reuseBased without its
    `mode = 2;` override) against the reference's own builder with that line
    removed: every partition's arrays, bit-exact."""
    by_name = {c["name"]: c for c in golden_cases}
    n = 0
    multi = 0
    for run in _heuristic_runs():
        dims, inds, vals = _inputs(by_name[run["case"]])
        got = O.build_mmcsf(dims, inds, vals, run["mode"], run["f"], partition="heuristic", fbth=run["h"])
        for k, v in run["arrays"].items():
            assert k in got, (run["case"], k)
            want = np.array(v, dtype=got[k].dtype)
            assert np.array_equal(got[k], want), (run["case"], run["h"], run["f"], k)
            n += 1
        multi += sum(int(run["arrays"][f"part{p}.nnz"][0]) > 0 for p in range(len(dims))) > 1
    assert n > 500 and multi >= 10


@pytest.mark.skipif(not O.ref_heur_available(), reason="reference oracle not built here")
@pytest.mark.parametrize("nd", [3, 4])
def test_partition_heuristic_matches_reference_library(nd, tmp_path):
    rng = np.random.default_rng(40 + nd)
    dims = [60, 90, 25] if nd == 3 else [20, 30, 12, 9]
    n = 4000
    inds = [np.minimum(rng.zipf(1.4, n) - 1, d - 1).astype(np.uint64) for d in dims]
    key = np.zeros(n, np.uint64)
    for m, d in enumerate(dims):
        key = key * np.uint64(d) + inds[m]
    _, first = np.unique(key, return_index=True)
    inds = [i[np.sort(first)] for i in inds]
    vals = (rng.random(len(inds[0])) + 0.1).astype(np.float32)
    p = str(tmp_path / "t.tns")
    O.write_tns(p, dims, inds, vals)
    dims2, inds2, vals2 = O.load_tns(p)
    for mode in range(nd):
        for h in (1, 3):
            ref = O.ref_dump_heuristic(p, mode, 5, h, str(tmp_path / "d.txt"))
            got = O.build_mmcsf(dims2, inds2, vals2, mode, 5, partition="heuristic", fbth=h)
            for k, v in ref.items():
                assert np.array_equal(got[k], v.astype(got[k].dtype)), (mode, h, k)
