"""mmcsf_sort_coo_noalloc: the construction sort with its scratch in a static
device array, for callers that cannot allocate device memory at run time.

Called through the C ABI on two tensors in a row (the second call must not
see anything the first left in the shared scratch); its output must equal,
bit for bit, the sorted nonzeros the allocating builder (mmcsf_build) exports
for the same format. Lives in its own file, collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NNZ = 1 << 19


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _coo(rng, dims, n, dup):
    inds = [rng.integers(0, d, n).astype(np.uint32) for d in dims]
    if not dup:
        key = np.zeros(n, np.uint64)
        for m, d in enumerate(dims):
            key = key * np.uint64(d) + inds[m].astype(np.uint64)
        _, first = np.unique(key, return_index=True)
        inds = [i[np.sort(first)] for i in inds]
    vals = (rng.random(len(inds[0])) + 0.5).astype(np.float32)
    return inds, vals


def _noalloc(torch, impl, mode, dims, inds, vals):
    from mmcsf import _lib
    nd = len(dims)
    n = len(vals)
    d_in = [torch.tensor(i.astype(np.int32), device="cuda") for i in inds]
    d_v = torch.tensor(vals, device="cuda")
    d_out = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(nd)]
    d_ov = torch.empty(n, dtype=torch.float32, device="cuda")
    P = ctypes.c_void_p
    st = _lib.lib().mmcsf_sort_coo_noalloc(
        impl, mode, nd, (ctypes.c_uint64 * nd)(*dims), ctypes.c_uint64(n),
        (P * nd)(*[P(t.data_ptr()) for t in d_in]), P(d_v.data_ptr()),
        (P * nd)(*[P(t.data_ptr()) for t in d_out]), P(d_ov.data_ptr()),
        P(torch.cuda.current_stream().cuda_stream))
    _lib.check(st)
    torch.cuda.synchronize()
    return [t.cpu().numpy().astype(np.uint64) for t in d_out], d_ov.cpu().numpy()


def _reference_order(impl, mode, dims, inds, vals):
    import mmcsf
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    F = mmcsf.Format(X, impl=impl, mode=mode, keep_coo=True)
    part = 2 if impl == mmcsf.IMPL_MMCSF else 0
    return [F.export(part, f"inds{m}") for m in range(len(dims))], F.export_f32(part, "vals")


@pytest.mark.parametrize("impl,mode", [(12, 0), (12, 2), (8, 1)])
def test_noalloc_sort_matches_builder_twice(impl, mode, torch_cuda):
    rng = np.random.default_rng(7 + impl + mode)
    # two calls in a row, different sizes and orders: 3-D then 4-D
    for dims, n, dup in (([400, 900, 120], 300_000, False), ([60, 50, 40, 30], 200_000, True)):
        inds, vals = _coo(rng, dims, n, dup)
        got_i, got_v = _noalloc(torch_cuda, impl, mode % len(dims), dims, inds, vals)
        want_i, want_v = _reference_order(impl, mode % len(dims), dims, inds, vals)
        for m in range(len(dims)):
            assert np.array_equal(got_i[m], want_i[m]), (impl, mode, dims, m)
        assert np.array_equal(got_v, want_v), (impl, mode, dims)


def test_noalloc_rejects_oversize(torch_cuda):
    from mmcsf import _lib
    P = ctypes.c_void_p
    dims = (ctypes.c_uint64 * 3)(10, 10, 10)
    dummy = torch_cuda.empty(4, device="cuda")
    ptrs = (P * 3)(*[P(dummy.data_ptr())] * 3)
    st = _lib.lib().mmcsf_sort_coo_noalloc(12, 0, 3, dims, ctypes.c_uint64(MAX_NNZ + 1), ptrs, P(dummy.data_ptr()),
                                           ptrs, P(dummy.data_ptr()), None)
    assert st == 1
    assert b"at most" in _lib.lib().mmcsf_last_error()
