"""Sharded one-tensor MTTKRP and CP-ALS across ranks (mmcsf.dist): every rank
owns a row range of every mode. Run as two and three gloo processes on the
CPU. The per-rank compute is the FP64 COO MTTKRP of the oracle on that rank's
shard of the mode (the CUDA kernels are covered by the GPU tests); what is
tested here is the sharding (ranges tile every mode, every nonzero in exactly
one shard per mode), the exchange (all-gather of owned rows, all-reduced
Grams and norms) and the replicated solve."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "mm-csf_b200"))

from mmcsf import dist as D  # noqa: E402
from oracle import cpals_oracle as CO  # noqa: E402


def _tensor(seed, dims=(30, 40, 25), nnz=3000, planted=0):
    rng = np.random.default_rng(seed)
    lin = rng.choice(int(np.prod(dims)), size=nnz, replace=False)
    inds = list(np.unravel_index(lin, dims))
    if planted:  # values of a planted rank-`planted` CP model
        A = [rng.random((d, planted)) for d in dims]
        p = np.ones((nnz, planted))
        for m in range(3):
            p *= A[m][inds[m]]
        vals = p.sum(1)
    else:
        vals = rng.random(nnz) + 0.1
    return list(dims), [np.asarray(i, np.int64) for i in inds], np.asarray(vals, np.float32)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _local_fn(sm, mode, factors):
    """This rank's rows of mode `mode` from the FP64 oracle on the rank's
    shard of that mode (the shard's mode index is rebased to the row range)."""
    lo, hi = sm.owned(mode)
    si, sv = sm.shards[mode]
    dims = list(sm.dims)
    dims[mode] = hi - lo
    U = [t.detach().cpu().numpy().astype(np.float64) for t in factors]
    U[mode] = np.zeros((hi - lo, U[mode].shape[1]))
    return torch.tensor(CO.mttkrp64(dims, si, sv, mode, U), dtype=torch.float32)


def _worker(rank, world, port, what, seed):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dims, inds, vals = _tensor(seed, planted=4 if what == "als" else 0)
        sm = D.ShardedMttkrp(dims, inds, vals, local_mttkrp=_local_fn)
        rng = np.random.default_rng(seed + 1)
        R = 4
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        Ut = [torch.tensor(u) for u in U]
        if what == "mttkrp":
            outs = sm.mttkrp_all(Ut)
            for m in range(3):
                want = CO.mttkrp64(dims, inds, vals, m, [u.astype(np.float64) for u in U])
                got = outs[m].numpy().astype(np.float64)
                assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max(), (rank, m)
                # without the gather: exactly this rank's rows, and no exchange needed
                lo, hi = sm.owned(m)
                part = sm.mttkrp(m, Ut, gather=False).numpy().astype(np.float64)
                assert part.shape[0] == hi - lo
                assert np.abs(part - want[lo:hi]).max() <= 1e-5 * np.abs(want).max(), (rank, m)
                # the ranks' row ranges tile the mode
                b = torch.tensor([lo, hi])
                allb = [torch.zeros_like(b) for _ in range(world)]
                dist.all_gather(allb, b)
                assert int(allb[0][0]) == 0 and int(allb[-1][1]) == dims[m]
                assert all(int(allb[r][1]) == int(allb[r + 1][0]) for r in range(world - 1))
                # every nonzero lives in exactly one rank's shard of each mode
                n = torch.tensor([sm.shard_nnz[m]])
                dist.all_reduce(n)
                assert int(n) == len(vals)
        else:
            Uo, lam_o, fit_o, hist_o = CO.cp_als(dims, inds, vals, U, max_iters=8, tol=1e-12)
            Ug, lam_g, fit_g, hist_g = D.dist_cp_als(sm, Ut, max_iters=8, tol=1e-12)
            assert len(hist_g) == len(hist_o)
            assert np.max(np.abs(np.array(hist_g) - np.array(hist_o))) <= 1e-5, (hist_g, hist_o)
            assert np.allclose(lam_g, lam_o, rtol=1e-3)
            # every rank holds the same factors
            for u in Ug:
                v = u.clone()
                dist.broadcast(v, 0)
                assert torch.equal(v, u)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("what", ["mttkrp", "als"])
def test_ranks_gloo(what, world):
    mp.spawn(_worker, args=(world, _free_port(), what, 3), nprocs=world, join=True)


def test_shard_slices_balance():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        counts = rng.zipf(1.5, size=500).clip(max=5000)
        b = D.shard_slices(counts, world)
        assert b[0] == 0 and b[-1] == len(counts) and all(x <= y for x, y in zip(b, b[1:]))
        loads = [int(counts[b[r]:b[r + 1]].sum()) for r in range(world)]
        assert sum(loads) == counts.sum()
        # each rank is within one slice of the even share
        assert max(loads) <= counts.sum() / world + counts.max()
    assert D.shard_slices([0, 0, 0], 2) == [0, 0, 3]
