"""TTM along the leaf mode (the reference's ttm, src/ttm.cu / ttm_cpu.cpp).

CPU: the oracle's TTM (oracle/mmcsf_oracle.c orc_ttm_f32) against the golden
outputs of the reference's own TTM_CPU (tests/golden/ttm.json) bit-exactly,
and against the reference library itself on fresh tensors when it is built.
GPU: mmcsf_ttm on a B-CSF format of each mode, FP32 and BF16 factors, with and
without fiber splits, against the oracle; the rows are the format's fibers."""
import json
import os
import sys
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import ttm_factor  # noqa: E402


def _case(name):
    with open(os.path.join(HERE, "golden", name + ".json")) as fh:
        c = json.load(fh)
    return c["dims"], [np.asarray(i, np.uint64) for i in c["inds"]], np.asarray(c["vals"], np.float32)


def test_ttm_oracle_vs_golden():
    with open(os.path.join(HERE, "golden", "ttm.json")) as fh:
        g = json.load(fh)
    assert g["runs"]
    for run in g["runs"]:
        dims, inds, vals = _case(run["case"])
        leaf = O.order_modes(dims, run["mode"])[2]
        u = ttm_factor(dims[leaf], g["R"])
        y, _, _ = O.ttm_f32(dims, inds, vals, run["mode"], u, run["f"] or O.INF_TH)
        want = np.asarray(run["Y"], np.float32).reshape(-1, g["R"])
        assert y.shape == want.shape and np.array_equal(y.view(np.uint32), want.view(np.uint32)), run["case"]


def test_ttm_oracle_vs_reference_library():
    if not O.ref_available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(3)
    for dims, n, f in (([30, 40, 20], 3000, 0), ([50, 8, 9], 2000, 2)):
        lin = rng.choice(int(np.prod(dims)), size=n, replace=False)
        inds = [np.asarray(i, np.uint64) for i in np.unravel_index(lin, dims)]
        vals = (rng.random(n) + 0.1).astype(np.float32)
        path = os.path.join(tempfile.mkdtemp(), "x.tns")
        O.write_tns(path, dims, inds, vals)
        for mode in range(3):
            u = rng.random((dims[O.order_modes(dims, mode)[2]], 16)).astype(np.float32)
            y, _, _ = O.ttm_f32(dims, inds, vals, mode, u, f or O.INF_TH)
            yr, nf = O.ref_ttm(path, mode, f, u, n + 2)
            assert nf == len(y) and np.array_equal(y, yr)


@pytest.mark.gpu
@pytest.mark.parametrize("R", [4, 16, 32, 64, 128])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_ttm_gpu_vs_oracle(R, dtype):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mmcsf
    rng = np.random.default_rng(R)
    for dims, n, skew in (([200, 300, 50], 20000, True), ([40, 30, 500], 8000, False)):
        if skew:
            inds = [np.minimum(rng.zipf(1.3, n) - 1, d - 1).astype(np.uint64) for d in dims]
        else:
            inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
        key = np.ravel_multi_index([i.astype(np.int64) for i in inds], dims)
        _, first = np.unique(key, return_index=True)
        first = np.sort(first)
        inds = [i[first] for i in inds]
        vals = (rng.random(len(first)) + 0.05).astype(np.float32)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        for mode in range(3):
            leaf = O.order_modes(dims, mode)[2]
            u = rng.random((dims[leaf], R)).astype(np.float32)
            ud = torch.tensor(u, device="cuda")
            if dtype == "bf16":
                ud = ud.to(torch.bfloat16)
                u = ud.float().cpu().numpy()
            for f in (0, 3):
                F = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=mode, fiber_threshold=f)
                got = F.ttm(ud).cpu().numpy().astype(np.float64)
                want, ptr, idx = O.ttm_f32(dims, inds, vals, mode, u, f or O.INF_TH)
                assert got.shape == want.shape, (mode, f)
                assert F.last_launches == 2  # main pass + side rows
                scale = np.abs(want).max()
                assert np.abs(got - want).max() <= 1e-5 * scale, (mode, f)
                # the rows are the format's fibers: its exported fiber indices are the oracle's
                assert np.array_equal(F.export(0, "fbrIdx1")[:len(want)], idx[1][:len(want)])
