"""Sampled CP model, its adjoint and gradient-based CP (Poisson loss).

* sampled model at every nonzero vs an FP64 numpy evaluation from the same
  factors (FP32 and BF16 factors, 3-D and 4-D, MM-CSF with and without views,
  B-CSF);
* adjoint (mmcsf_cp_adjoint) vs the reference's own MTTKRP_COO_CPU run on the
  same sparsity with the upstream gradients as values (oracle/_ref), and vs
  the FP64 COO MTTKRP of the oracle;
* autograd gradients of the Poisson loss vs FP64 central finite differences
  (eps = 1e-3) and vs the gradient assembled from the reference's MTTKRP;
* projected-Adam Poisson CP: loss falls, BF16 factors track FP32.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _bf16_round(a):
    """Round-to-nearest-even to BF16, returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def _model64(coords, factors, lam=None):
    R = factors[0].shape[1]
    p = np.ones((len(coords[0]), R))
    for c, f in zip(coords, factors):
        p *= f.astype(np.float64)[c.astype(np.int64)]
    if lam is not None:
        p *= lam.astype(np.float64)
    return p.sum(1)


def _build(dims, nnz, seed, impl, mode=0, views=0, fbr_th=0, zipf=False, poisson=False, planted=0):
    import mmcsf
    X = mmcsf.CooTensor.generate(dims, nnz, dist=[1 if zipf else 0] * len(dims), zipf_s=1.05,
                                 val_dist=mmcsf.VAL_UNIFORM01, seed=seed, planted_rank=planted,
                                 poisson=poisson)
    F = mmcsf.Format(X, impl=impl, mode=mode, fiber_threshold=fbr_th, keep_coo=True, views=views)
    return X, F


CASES = [
    # (dims, nnz, impl, mode, views, fbr_th)
    ([300, 200, 100], 20000, 12, 0, 0, 0),
    ([300, 200, 100], 20000, 12, 0, 1, 8),
    ([60, 50, 40, 30], 30000, 12, 0, 1, 0),
    ([60, 50, 40, 30], 30000, 12, 0, 0, 16),
    ([300, 200, 100], 20000, 8, 1, 0, 16),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("R", [4, 32, 256])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_sampled_model_vs_fp64(case, R, dtype, torch_cuda):
    torch = torch_cuda
    import mmcsf
    dims, nnz, impl, mode, views, fth = case
    X, F = _build(dims, nnz, seed=R + len(dims), impl=impl, mode=mode, views=views, fbr_th=fth, zipf=True)
    rng = np.random.default_rng(R)
    U = [rng.random((d, R)).astype(np.float32) for d in dims]
    lam = rng.random(R).astype(np.float32) + 0.5
    if dtype == "bf16":
        U = [_bf16_round(u) for u in U]
    tdt = torch.bfloat16 if dtype == "bf16" else torch.float32
    Ud = [torch.tensor(u, device="cuda").to(tdt) for u in U]
    got = F.sampled_model(Ud, torch.tensor(lam, device="cuda")).cpu().numpy().astype(np.float64)
    coords = F.nonzero_coords()
    want = _model64(coords, U, lam)
    assert got.shape == want.shape == (F.nnz,)
    err = np.max(np.abs(got - want) / np.abs(want))
    assert err <= 2e-6 * np.sqrt(R), err
    # lambda = None is all ones
    got1 = F.sampled_model(Ud).cpu().numpy().astype(np.float64)
    assert np.max(np.abs(got1 - _model64(coords, U)) / _model64(coords, U)) <= 2e-6 * np.sqrt(R)
    assert F.last_launches == 1
    # values() and the nonzero order agree with the tensor's (coordinate, value) pairs
    inds, vals = X.host_arrays()
    key = lambda cs: np.ravel_multi_index([c.astype(np.int64) for c in cs], dims)  # noqa: E731
    a = dict(zip(key(inds).tolist(), vals.tolist()))
    v = F.values().cpu().numpy()
    assert all(a[k] == x for k, x in zip(key(coords).tolist(), v.tolist()))


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("R", [8, 32, 100])
def test_adjoint_vs_reference_mttkrp(case, R, torch_cuda):
    torch = torch_cuda
    dims, nnz, impl, mode, views, fth = case
    X, F = _build(dims, nnz, seed=7 * R, impl=impl, mode=mode, views=views, fbr_th=fth, zipf=True)
    rng = np.random.default_rng(R + 1)
    U = [rng.random((d, R)).astype(np.float32) for d in dims]
    lam = rng.random(R).astype(np.float32) + 0.5
    grad = (rng.random(F.nnz) - 0.5).astype(np.float32)
    Ud = [torch.tensor(u, device="cuda") for u in U]
    coords = F.nonzero_coords()
    modes = range(len(dims)) if impl == 12 else [mode]
    for n in modes:
        got = F.cp_adjoint(n, Ud, torch.tensor(grad, device="cuda"), torch.tensor(lam, device="cuda"))
        got = got.cpu().numpy().astype(np.float64)
        want64 = O.mttkrp_coo_f64(dims, coords, grad, n, U) * lam
        scale = np.abs(want64).max()
        assert np.abs(got - want64).max() <= 1e-5 * scale
        if O.ref_available():
            want_ref = O.ref_mttkrp_coo(dims, coords, grad, n, U).astype(np.float64) * lam
            assert np.abs(got - want_ref).max() <= 1e-5 * scale
        # lambda omitted: plain MTTKRP on the gradient values
        plain = F.cp_adjoint(n, Ud, torch.tensor(grad, device="cuda")).cpu().numpy()
        assert np.abs(plain - want64 / lam).max() <= 1e-5 * np.abs(want64 / lam).max()


def _poisson64(coords, y, factors, eps=1e-10):
    cs = np.ones(factors[0].shape[1])
    for f in factors:
        cs *= f.sum(0)
    return cs.sum() - np.sum(y * np.log(_model64(coords, factors) + eps))


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
@pytest.mark.parametrize("views", [0, 1])
def test_poisson_gradient_fd_and_reference(precision, views, torch_cuda):
    torch = torch_cuda
    from mmcsf import gcp
    dims = [14, 11, 9]
    R = 4
    X, F = _build(dims, 400, seed=5 + views, impl=12, views=views, poisson=True, planted=3)
    coords = F.nonzero_coords()
    y = F.values().cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(11)
    U = [_bf16_round(0.5 + rng.random((d, R)).astype(np.float32)) for d in dims]
    masters = [torch.tensor(u, device="cuda", requires_grad=True) for u in U]
    loss = gcp.poisson_loss(F, masters, F.values(), precision=precision)
    loss.backward()
    gots = [m.grad.cpu().numpy().astype(np.float64) for m in masters]
    U64 = [u.astype(np.float64) for u in U]
    assert abs(loss.item() - _poisson64(coords, y, U64)) <= 1e-5 * abs(_poisson64(coords, y, U64))
    eps = 1e-3
    for n in range(3):
        scale = np.abs(gots[n]).max()
        for i, r in zip(rng.integers(0, dims[n], 12), rng.integers(0, R, 12)):
            up = [u.copy() for u in U64]
            dn = [u.copy() for u in U64]
            up[n][i, r] += eps
            dn[n][i, r] -= eps
            fd = (_poisson64(coords, y, up) - _poisson64(coords, y, dn)) / (2 * eps)
            assert abs(gots[n][i, r] - fd) <= 1e-4 * max(scale, abs(fd)), (n, i, r, gots[n][i, r], fd)
    # the gradient assembled from the reference's own MTTKRP_COO_CPU
    w = -(y / (_model64(coords, U64) + 1e-10))
    for n in range(3):
        cs = np.ones(R)
        for m in range(3):
            if m != n:
                cs *= U64[m].sum(0)
        mk = O.ref_mttkrp_coo(dims, coords, w.astype(np.float32), n, U) if O.ref_available() else \
            O.mttkrp_coo_f64(dims, coords, w.astype(np.float32), n, U)
        want = cs[None, :] + mk.astype(np.float64)
        assert np.abs(gots[n] - want).max() <= 1e-5 * np.abs(want).max()


def test_lambda_gradient(torch_cuda):
    torch = torch_cuda
    from mmcsf import gcp
    dims = [40, 30, 20]
    R = 8
    X, F = _build(dims, 3000, seed=3, impl=12, views=1)
    rng = np.random.default_rng(4)
    U = [rng.random((d, R)).astype(np.float32) for d in dims]
    lam = (rng.random(R) + 0.5).astype(np.float32)
    w = (rng.random(F.nnz) - 0.5).astype(np.float32)
    Ud = [torch.tensor(u, device="cuda", requires_grad=True) for u in U]
    ld = torch.tensor(lam, device="cuda", requires_grad=True)
    xhat = gcp.sampled_cp(F, Ud, ld)
    (xhat * torch.tensor(w, device="cuda")).sum().backward()
    coords = F.nonzero_coords()
    # d/dlam_r sum_x w_x xhat_x = sum_x w_x prod_m A_m[i_m, r]
    p = np.ones((F.nnz, R))
    for c, u in zip(coords, U):
        p *= u.astype(np.float64)[c.astype(np.int64)]
    want = (w.astype(np.float64)[:, None] * p).sum(0)
    assert np.abs(ld.grad.cpu().numpy() - want).max() <= 1e-5 * np.abs(want).max()
    for n in range(3):
        want_n = O.mttkrp_coo_f64(dims, coords, w, n, U) * lam
        assert np.abs(Ud[n].grad.cpu().numpy() - want_n).max() <= 1e-5 * np.abs(want_n).max()


def test_gcp_poisson_bf16_tracks_fp32(torch_cuda):
    from mmcsf import gcp
    dims = [2000, 1000, 500]
    X, F = _build(dims, 200000, seed=21, impl=12, views=1, zipf=True, poisson=True, planted=8)
    runs = {p: gcp.gcp_poisson(F, 8, iters=60, lr=0.05, precision=p, seed=1) for p in ("fp32", "bf16")}
    for p, r in runs.items():
        assert r["iters"] == 60
        assert r["loss"][-1] < r["loss"][0]
        assert all(b >= a for a, b in zip(r["ms"], r["ms"][1:]))
        for f in r["factors"]:
            assert float(f.min()) >= 0.0
    l32, l16 = runs["fp32"]["loss"][-1], runs["bf16"]["loss"][-1]
    assert abs(l16 - l32) <= 1e-3 * abs(l32), (l32, l16)


@pytest.mark.parametrize("impl,views", [(12, 0), (12, 1), (12, 2)])
@pytest.mark.parametrize("R", [8, 32, 64])
@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_fused_poisson_step_matches_unfused(impl, views, R, precision, torch_cuda):
    """The one-pass Poisson kernel (model, w = y/(xhat+eps), loss, slice-mode
    gradient) gives the loss and every factor gradient of the sampled model +
    torch ops + adjoints path."""
    torch = torch_cuda
    from mmcsf import gcp
    dims = [700, 400, 90]
    X, F = _build(dims, 60000, seed=R, impl=impl, mode=0, views=views, zipf=True, poisson=True, planted=4)
    rng = np.random.default_rng(R)
    U = [_bf16_round(0.2 + rng.random((d, R)).astype(np.float32)) for d in dims]
    res = {}
    for fused in (False, True):
        masters = [torch.tensor(u, device="cuda", requires_grad=True) for u in U]
        loss = gcp.poisson_loss(F, masters, F.values(), precision=precision, fused=fused)
        loss.backward()
        res[fused] = (float(loss.detach()), [m.grad.double().cpu().numpy() for m in masters])
    l0, g0 = res[False]
    l1, g1 = res[True]
    assert abs(l1 - l0) <= 1e-5 * abs(l0), (l0, l1)
    for a, b in zip(g0, g1):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max()
    # one launch computes the model, the loss and the slice-mode gradient
    w, g_root, lz, root = F.poisson_step([torch.tensor(u, device="cuda") for u in U])
    assert F.last_launches == 1 and w.shape == (F.nnz,) and g_root.shape[0] == dims[root]
