"""Parity at the benchmarked shapes.

* The 1000 x 1000 x 1000, 100,000-nonzero uniform tensor with -f 128 (the
  metric's first configuration, as the benchmark generates it): every MM-CSF
  array bit-exact against the oracle's replay of the reference's builders, and
  every mode's MTTKRP element by element within 1e-5 of the FP64 oracle, for
  the -w 1 mapping, the default and the tuned plans.
* A tensor of the skewed 500,000 x 2,000,000 x 20,000 shape (Zipf(1.1) per
  mode, lognormal values) at 3M nonzeros: arrays bit-exact, and at R = 32 and
  R = 64 every traversal the tuner can pick (partition or view, kernels 1-4,
  every occupancy level) and the two-output walks element by element within
  1e-5 of the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from test_gpu_parity import _check_close, _compare_dumps

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_config1_exact(torch_cuda):
    torch = torch_cuda
    import mmcsf
    dims = [1000, 1000, 1000]
    X = mmcsf.CooTensor.generate(dims, 100_000, dist=[0, 0, 0], val_dist=mmcsf.VAL_UNIFORM01, seed=0)
    inds, vals = X.host_arrays()
    inds = [i.astype(np.uint64) for i in inds]
    ref = O.build_mmcsf(dims, inds, vals, 0, 128)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=128, keep_coo=True, views=1)
    _compare_dumps(ref, F.reference_dump(), "mmcsf", 3, "config1")
    R = 32
    rng = np.random.default_rng(0)
    U = [rng.random((d, R)).astype(np.float32) for d in dims]
    Ud = [torch.tensor(u, device="cuda") for u in U]
    want = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(3)]
    cfg = {"chunk": F.chunk_for_warps(1, R)}
    for m in range(3):
        _check_close(F.mttkrp(m, Ud, cfg=cfg).cpu().numpy(), want[m], ("-w 1", m))
    outs = F.mttkrp_all(Ud)
    for m in range(3):
        _check_close(outs[m].cpu().numpy(), want[m], ("default", m))
    F.tune(Ud)
    outs = F.mttkrp_all(Ud)
    for m in range(3):
        _check_close(outs[m].cpu().numpy(), want[m], ("tuned", m))


@pytest.fixture(scope="module")
def skewed(torch_cuda):
    import mmcsf
    dims = [500000, 2000000, 20000]
    X = mmcsf.CooTensor.generate(dims, 3_000_000, dist=[1, 1, 1], zipf_s=1.1, val_dist=mmcsf.VAL_LOGNORMAL, seed=7)
    inds, vals = X.host_arrays()
    return dims, X, [i.astype(np.uint64) for i in inds], vals


def test_skewed_shape_arrays_bit_exact(skewed):
    import mmcsf
    dims, X, inds, vals = skewed
    ref = O.build_mmcsf(dims, inds, vals, 0, O.INF_TH)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, keep_coo=True)
    _compare_dumps(ref, F.reference_dump(), "mmcsf", 3, "skewed 3M")


@pytest.mark.parametrize("R", [32, 64])
def test_skewed_shape_every_traversal(R, skewed, torch_cuda):
    torch = torch_cuda
    import mmcsf
    dims, X, inds, vals = skewed
    rng = np.random.default_rng(R)
    U = [rng.random((d, R)).astype(np.float32) for d in dims]
    Ud = [torch.tensor(u, device="cuda") for u in U]
    want = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(3)]
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, views=2)
    for m in range(3):
        for trav in ((1, 2) if F.info(4 + m)["present"] else (1,)):  # the partition's slice mode has no view
            for kern in (1, 2, 3, 4, 5, 6, 7):
                for mb in (1, 2, 3, 4):
                    cfg = {"traversal": trav, "kernel": kern, "min_blocks": mb, "chunk": 512}
                    _check_close(F.mttkrp(m, Ud, cfg=cfg).cpu().numpy(), want[m], (R, m, cfg))
    m0, m1 = F.pair_modes()
    for kern in (2, 3, 4, 5, 6, 7):
        for mb in (1, 2, 3, 4):
            outs = F.mttkrp_pair(Ud, cfg={"kernel": kern, "min_blocks": mb, "chunk": 512})
            for m in (m0, m1):
                _check_close(outs[m].cpu().numpy(), want[m], ("pair", R, kern, mb, m))
    F.tune(Ud)
    outs = F.mttkrp_all(Ud)
    for m in range(3):
        _check_close(outs[m].cpu().numpy(), want[m], ("tuned", R, m))
