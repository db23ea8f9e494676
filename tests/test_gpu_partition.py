"""The MM-CSF partition heuristic on the device (partition_rule=1): the
reference's mm_partition_reuseBased without its `mode = 2;` override.

* partitions: every array of every partition bit-exact against the
  reference's own builder with that line removed (tests/golden/heuristic.json)
  and against the oracle's sequential restatement on fresh tensors;
* MTTKRP, CP-ALS and the sampled model over several partitions: within the
  FP64-oracle tolerance of the parity tests.
"""
import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_parity import _check_close, _rand_coo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _compare(ref, got, nd, ctx):
    """Every reference array, exactly; a partition's leaf-level sentinel only
    where the reference defines it (it reads one past the partition's last
    nonzero when the last fiber holds two or more)."""
    for k, v in ref.items():
        assert k in got, (ctx, k)
        g = got[k]
        if k.endswith("vals"):
            assert np.array_equal(np.asarray(v, np.float32), g), (ctx, k)
            continue
        v = np.asarray(v).astype(np.int64)
        g = np.asarray(g).astype(np.int64)
        pfx = k.split(".")[0]
        if k == f"{pfx}.fbrIdx{nd - 2}" and len(v):
            ptr = np.asarray(ref[f"{pfx}.fbrPtr{nd - 2}"], np.int64)
            defined = len(ptr) < 2 or ptr[-1] - ptr[-2] == 1 or int(ref[f"{pfx}.nnz"][0]) == 1
            assert len(v) == len(g) and np.array_equal(v[:-1], g[:-1]), (ctx, k)
            if defined:
                assert v[-1] == g[-1], (ctx, k, "sentinel")
            continue
        assert len(v) == len(g) and np.array_equal(v, g), (ctx, k, v[:12], g[:12])


def _heuristic_runs():
    import json
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    with open(os.path.join(here, "heuristic.json")) as fh:
        return json.load(fh)["runs"]


def test_golden_partitions_bit_exact(golden_cases, torch_cuda):
    import mmcsf
    by_name = {c["name"]: c for c in golden_cases}
    n = multi = 0
    for run in _heuristic_runs():
        case = by_name[run["case"]]
        dims = case["dims"]
        X = mmcsf.CooTensor.from_arrays(dims, case["inds"], case["vals"])
        F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=run["mode"], fiber_threshold=run["f"], keep_coo=True,
                         partition_rule=1, partition_ratio=run["h"])
        _compare(run["arrays"], F.reference_dump(), len(dims), (run["case"], run["h"], run["f"]))
        n += 1
        multi += len(F.partitions()) > 1
    assert n >= 25 and multi >= 10


CASES = [
    # nd, dims, nnz, skew, f, ratio
    (3, [300, 500, 200], 20000, False, 0, 1),
    (3, [300, 500, 200], 20000, True, 4, 1),
    (3, [64, 2000, 40], 30000, True, 0, 2),
    (3, [60, 60, 60], 20000, True, 2, 3),
    (4, [200, 40, 30, 10], 30000, False, 0, 1),
    (4, [300, 20, 10, 6], 30000, True, 3, 1),
    (4, [50, 40, 30, 20], 30000, True, 0, 2),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_random_partitions_match_oracle(case, torch_cuda):
    import mmcsf
    nd, dims, n, skew, f, ratio = CASES[case]
    rng = np.random.default_rng(700 + case)
    inds, vals = _rand_coo(rng, dims, n, skew)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    fth = f if f else O.INF_TH
    for mode in range(nd):
        ref = O.build_mmcsf(dims, inds, vals, mode, fth, partition="heuristic", fbth=ratio)
        F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=mode, fiber_threshold=f, keep_coo=True, partition_rule=1,
                         partition_ratio=ratio)
        _compare(ref, F.reference_dump(), nd, (case, mode))
        assert sum(F.info(p)["nnz"] for p in F.partitions()) == len(vals)


def test_large_skewed_partitions_match_oracle(torch_cuda):
    """2M nonzeros, Zipf(1.1) in every mode: the partition of every nonzero
    (through the partitions' coordinates) equals the sequential oracle's."""
    import mmcsf
    dims = [50000, 200000, 2000]
    X = mmcsf.CooTensor.generate(dims, 2_000_000, dist=[1, 1, 1], zipf_s=1.1, val_dist=mmcsf.VAL_LOGNORMAL, seed=3)
    inds, vals = X.host_arrays()
    inds = [np.asarray(i, np.uint64) for i in inds]
    vals = np.asarray(vals, np.float32)
    ref = O.build_mmcsf(dims, inds, vals, 0, O.INF_TH, partition="heuristic")
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, keep_coo=True, partition_rule=1)
    rule, rounds = F.partitioning()
    assert rule == 1 and 1 <= rounds <= 50, rounds
    got = F.reference_dump()
    counts = [int(ref[f"part{p}.nnz"][0]) for p in range(3)]
    assert sum(c > 0 for c in counts) >= 2, counts
    for p in range(3):
        assert int(got[f"part{p}.nnz"][0]) == counts[p], (p, counts)
        for m in range(3):
            if counts[p]:
                assert np.array_equal(got[f"part{p}.inds{m}"].astype(np.uint64), ref[f"part{p}.inds{m}"]), (p, m)


@pytest.mark.parametrize("nd", [3, 4])
@pytest.mark.parametrize("views", [0, 1, 2])
def test_mttkrp_over_partitions(nd, views, torch_cuda):
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(800 + nd * 10 + views)
    dims = [150, 400, 60] if nd == 3 else [60, 50, 40, 30]
    inds, vals = _rand_coo(rng, dims, 30000, True)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=4, views=views, partition_rule=1)
    assert len(F.partitions()) > 1
    for R in (8, 32, 48):
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        Ud = [torch.tensor(u, device="cuda") for u in U]
        ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(nd)]
        outs = F.mttkrp_all(Ud)
        for m in range(nd):
            _check_close(outs[m].cpu().numpy(), ref[m], ("all", nd, views, R, m))
            for kern in (1, 2, 3):
                for trav in ((1, 2) if views and F.info(4 + m)["present"] else (1,)):
                    out = F.mttkrp(m, Ud, cfg={"kernel": kern, "traversal": trav})
                    _check_close(out.cpu().numpy(), ref[m], ("mode", nd, views, R, m, kern, trav))
        if R == 32:
            F.tune(Ud)
            outs = F.mttkrp_all(Ud)
            for m in range(nd):
                _check_close(outs[m].cpu().numpy(), ref[m], ("tuned", nd, views, m))
            houts = F.mttkrp_all_host(U)
            for m in range(nd):
                _check_close(houts[m], ref[m], ("host", nd, views, m))
            Ub = [t.to(torch.bfloat16) for t in Ud]
            Ubf = [t.float().cpu().numpy() for t in Ub]
            outs = F.mttkrp_all(Ub)
            for m in range(nd):
                _check_close(outs[m].cpu().numpy(), O.mttkrp_coo_f64(dims, inds, vals, m, Ubf), ("bf16", nd, m))


def test_sampled_model_and_adjoint_over_partitions(torch_cuda):
    """Values, coordinates, the sampled model and its adjoint all use the
    format's nonzero order (partitions 0..nd-1)."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(900)
    dims = [150, 400, 60]
    inds, vals = _rand_coo(rng, dims, 30000, True)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    for views in (0, 2):
        F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, keep_coo=True, views=views, partition_rule=1)
        assert len(F.partitions()) > 1
        coords = F.nonzero_coords()
        fv = F.values().cpu().numpy()
        key = lambda c: (c[0].astype(np.int64) * dims[1] + c[1]) * dims[2] + c[2]  # noqa: E731
        order = np.argsort(key(coords))
        ref_order = np.argsort(key([np.asarray(i, np.int64) for i in inds]))
        assert np.array_equal(key(coords)[order], key([np.asarray(i, np.int64) for i in inds])[ref_order])
        assert np.array_equal(fv[order], np.asarray(vals, np.float32)[ref_order])
        R = 16
        A = [rng.random((d, R)).astype(np.float32) for d in dims]
        Ad = [torch.tensor(a, device="cuda") for a in A]
        xhat = F.sampled_model(Ad).cpu().numpy().astype(np.float64)
        want = np.ones((len(fv), R))
        for m in range(3):
            want *= A[m][coords[m].astype(np.int64)]
        assert np.allclose(xhat, want.sum(1), rtol=1e-5, atol=1e-6)
        g = rng.random(len(fv)).astype(np.float32)
        gd = torch.tensor(g, device="cuda")
        for m in range(3):
            out = F.cp_adjoint(m, Ad, gd).cpu().numpy()
            ref = O.mttkrp_coo_f64(dims, [c.astype(np.uint64) for c in coords], g, m, A)
            _check_close(out, ref, ("adjoint", views, m))


def test_cpals_over_partitions(torch_cuda):
    """CP-ALS on a heuristic-partitioned format follows the same iterates as
    on the shipped single-partition format (same tensor, same start)."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(950)
    dims = [200, 300, 100]
    inds, vals = _rand_coo(rng, dims, 40000, True)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    init = [torch.tensor(rng.random((d, 8)).astype(np.float32), device="cuda") for d in dims]
    runs = []
    for rule in (0, 1):
        # no views: the loop walks one mode at a partition's leaf level, whose FP64
        # scratch mmcsf_cpd allocates before it captures the loop into a graph
        F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, partition_rule=rule)
        runs.append(F.cpd(8, max_iters=6, tol=0, precision="fp32", init=init))
        assert runs[-1]["graph"]
        h = F.cpd(8, max_iters=6, tol=0, precision="fp32", init=init, graph=False)
        assert np.max(np.abs(np.array(h["history"]) - np.array(runs[-1]["history"]))) <= 1e-6
        b = F.cpd(8, max_iters=6, tol=0, precision="bf16", init=init)  # the BF16 form's graph on the same format
        assert b["graph"] and b["iters"] == 6
        assert abs(b["history"][-1] - runs[-1]["history"][-1]) <= 1e-2, (b["history"], runs[-1]["history"])
    h0, h1 = np.array(runs[0]["history"]), np.array(runs[1]["history"])
    assert len(h0) == len(h1)
    assert np.max(np.abs(h0 - h1)) <= 1e-4, (h0, h1)


def test_heuristic_refuses_out_of_bounds_inputs(torch_cuda):
    """One slice holding several fibers in a mode's CSF: the reference's
    lookup reads before its arrays there, so both sides refuse."""
    import mmcsf
    dims = [1, 6, 7]
    rng = np.random.default_rng(3)
    inds, vals = _rand_coo(rng, dims, 30)
    with pytest.raises(ValueError):
        O.build_mmcsf(dims, inds, vals, 0, O.INF_TH, partition="heuristic")
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, partition_rule=1)
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, partition_rule=1)
