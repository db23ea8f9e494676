"""mmcsf_format_check on the GPU: every format kind the library builds passes
it; factors with fewer rows than a mode's indices need are reported (the
check only reads the format's arrays); and the bounds-checked library
(lib/libmmcsf_bounds.so, every compute entry point validating its format
first) runs the MTTKRP, CP-ALS and TTM paths with the same results."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _coo(rng, dims, n, skew):
    if skew:
        inds = [np.minimum(rng.zipf(1.4, n) - 1, d - 1).astype(np.uint64) for d in dims]
    else:
        inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    key = np.zeros(n, np.uint64)
    for m, d in enumerate(dims):
        key = key * np.uint64(d) + inds[m]
    _, first = np.unique(key, return_index=True)
    first = np.sort(first)
    inds = [i[first] for i in inds]
    return inds, (rng.random(len(inds[0])) + 0.05).astype(np.float32)


CASES = [([150, 400, 60], 20000, True), ([3000, 50, 40], 9000, False), ([40, 30, 50, 20], 20000, True),
         ([900, 8, 6, 5], 6000, False), ([5, 7, 900], 3000, False)]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_every_format_passes(case, torch_cuda):
    import mmcsf
    dims, n, skew = CASES[case]
    rng = np.random.default_rng(900 + case)
    inds, vals = _coo(rng, dims, n, skew)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    for f in (0, 3):
        for views in (0, 2):
            mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f, views=views).check()
        mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, partition_rule=1, fiber_threshold=f).check()
        for m in range(len(dims)):
            mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=m, fiber_threshold=f).check()
            mmcsf.Format(X, impl=mmcsf.IMPL_HBCSF, mode=m, fiber_threshold=f).check()
        mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=2).check(rows=dims)


def test_short_factor_reported(torch_cuda):
    import mmcsf
    rng = np.random.default_rng(5)
    dims = [150, 400, 60]
    inds, vals = _coo(rng, dims, 20000, False)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, views=2)
    F.check(rows=dims)
    for m in range(3):
        rows = list(dims)
        rows[m] = int(inds[m].max())  # one row short of the largest index of mode m
        with pytest.raises(mmcsf.MmcsfError, match=f"mode {m}"):
            F.check(rows=rows)
    H = mmcsf.Format(X, impl=mmcsf.IMPL_HBCSF, mode=1)
    with pytest.raises(mmcsf.MmcsfError, match="format check"):
        H.check(rows=[1, 1, 1])


_CHILD = r"""
import os, sys, json
import numpy as np
sys.path[:0] = [os.environ["ROOT"], os.path.join(os.environ["ROOT"], "mm-csf_b200")]
import torch, mmcsf
from mmcsf import _lib
from oracle import oracle as O
assert _lib.LIB_PATH.endswith("libmmcsf_bounds.so"), _lib.LIB_PATH
dims = [300, 400, 50]
X = mmcsf.CooTensor.generate(dims, 40000, dist=[1, 1, 1], zipf_s=1.1, val_dist=mmcsf.VAL_LOGNORMAL, seed=3)
inds, vals = X.host_arrays()
inds = [i.astype(np.uint64) for i in inds]
rng = np.random.default_rng(1)
U = [rng.random((d, 32)).astype(np.float32) for d in dims]
Ud = [torch.tensor(u, device="cuda") for u in U]
err = {}
for impl in (mmcsf.IMPL_MMCSF, mmcsf.IMPL_BCSF, mmcsf.IMPL_HBCSF):
    F = mmcsf.Format(X, impl=impl, mode=1, views=2 if impl == mmcsf.IMPL_MMCSF else 0)
    modes = range(3) if impl == mmcsf.IMPL_MMCSF else [1]
    for m in modes:
        got = F.mttkrp(m, Ud).double().cpu().numpy()
        ref = O.mttkrp_coo_f64(dims, inds, vals, m, U)
        err[f"{impl}_{m}"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=2)
r = F.cpd(8, max_iters=3, tol=0.0)
err["cpd_iters"] = r["iters"]
print(json.dumps(err))
"""


def test_bounds_checked_library(torch_cuda):
    lib = os.path.join(ROOT, "mm-csf_b200", "lib", "libmmcsf_bounds.so")
    assert os.path.exists(lib)
    env = dict(os.environ, MMCSF_LIBRARY=lib, ROOT=ROOT)
    r = subprocess.run([sys.executable, "-c", _CHILD], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    import json
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res.pop("cpd_iters") == 3
    for k, v in res.items():
        assert v <= 1e-5, (k, v)
