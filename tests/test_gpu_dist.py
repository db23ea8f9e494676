"""The sharded path's per-rank compute on the GPU (one rank: every mode's
shard is the whole tensor, one B-CSF of the mode each): ShardedMttkrp through
the CUDA library against the FP64 oracle, from host and from device arrays,
tuned; and dist_cp_als against the FP64 ALS restatement."""
import numpy as np
import pytest

from oracle import cpals_oracle as CO
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_sharded_single_rank_cuda(torch_cuda):
    torch = torch_cuda
    import mmcsf
    from mmcsf import dist as D
    dims = [60, 80, 50]
    X = mmcsf.CooTensor.generate(dims, 20000, dist=[1, 1, 1], zipf_s=1.1, seed=9, planted_rank=4, noise=0.01)
    inds, vals = X.host_arrays()
    sm = D.ShardedMttkrp(dims, inds, vals)
    assert all(f is not None for f in sm.fmts) and sm.shard_nnz == [len(vals)] * 3
    assert sm.rows == [(0, d) for d in dims]
    rng = np.random.default_rng(1)
    U = [rng.random((d, 8)).astype(np.float32) for d in dims]
    Ud = [torch.tensor(u, device="cuda") for u in U]
    want = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(3)]
    di, dv = X.device_tensors()
    smd = D.ShardedMttkrp(dims, [i.clone() for i in di], dv.clone(), device="cuda")
    for s_ in (sm, smd):
        for tuned in (False, True):
            if tuned:
                s_.tune(Ud)
            outs = s_.mttkrp_all(Ud)
            for m in range(3):
                assert np.abs(outs[m].cpu().numpy() - want[m]).max() <= 1e-5 * np.abs(want[m]).max(), (m, tuned)
    Ug, lam, fit, hist = D.dist_cp_als(sm, Ud, max_iters=6, tol=1e-12)
    Uo, lam_o, fit_o, hist_o = CO.cp_als(dims, [i.astype(np.int64) for i in inds], vals, U, max_iters=6, tol=1e-12)
    assert np.max(np.abs(np.array(hist) - np.array(hist_o))) <= 1e-4
