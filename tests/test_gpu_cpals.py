"""CP-ALS on the device (mmcsf_cpd) against the FP64 restatement of the
reference's cpd() (oracle/cpals_oracle.py), started from the same factors.

* FP32 form: fit history within 1e-4 of FP64 and normalised factors/lambda
  close; the FP64-solve form tighter (1e-6 on the fit);
* BF16 form (BF16 factors, FP64 Gram/solve/fit, the whole loop in one CUDA
  graph): on a planted low-rank tensor it converges to the FP64 run's fit
  within 1e-4, and the graph and host-driven runs agree;
* every form: the one-graph loop and the host-driven loop give the same fit
  history; on the default stream the FP32 forms run host-driven.
"""
import numpy as np
import pytest

from oracle import cpals_oracle as CO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _tensor(dims, nnz, seed, planted=0, noise=0.0):
    import mmcsf
    X = mmcsf.CooTensor.generate(dims, nnz, dist=[0] * len(dims), val_dist=mmcsf.VAL_UNIFORM01, seed=seed,
                                 planted_rank=planted, noise=noise)
    inds, vals = X.host_arrays()
    return X, [i.astype(np.int64) for i in inds], vals


def _init(torch, dims, R, seed):
    g = np.random.default_rng(seed)
    U = [g.random((d, R)).astype(np.float32) for d in dims]
    return U, [torch.tensor(u, device="cuda") for u in U]


@pytest.mark.parametrize("R", [4, 8, 16])
@pytest.mark.parametrize("precision,tol", [("fp32", 1e-4), ("fp64solve", 1e-6)])
def test_cpd_tracks_fp64_oracle(R, precision, tol, torch_cuda):
    import mmcsf
    dims = [40, 55, 30]
    X, inds, vals = _tensor(dims, 6000, seed=R)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=1)
    U, Ud = _init(torch_cuda, dims, R, seed=100 + R)
    res = F.cpd(R, max_iters=6, tol=0.0 + 1e-12, precision=precision, init=Ud)
    Uo, lam_o, fit_o, hist_o = CO.cp_als(dims, inds, vals, U, max_iters=6, tol=1e-12)
    assert res["iters"] == len(hist_o) == 6
    assert np.max(np.abs(np.array(res["history"]) - np.array(hist_o))) <= tol, (res["history"], hist_o)
    # final factors are column-normalised; compare the rank-one components
    for m in range(3):
        got = res["factors"][m].cpu().numpy().astype(np.float64)
        assert np.linalg.norm(got - Uo[m]) / np.linalg.norm(Uo[m]) <= (5e-3 if precision == "fp32" else 1e-4)
    assert np.allclose(res["lambda"], lam_o, rtol=(5e-3 if precision == "fp32" else 1e-4))


def test_cpd_bf16_graph_reaches_fp64_fit(torch_cuda):
    import mmcsf
    dims = [120, 150, 90]
    X, inds, vals = _tensor(dims, 40000, seed=5, planted=4, noise=0.01)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=1)
    U, Ud = _init(torch_cuda, dims, 4, seed=9)
    _, _, fit_o, hist_o = CO.cp_als(dims, inds, vals, U, max_iters=50, tol=1e-5)
    g = F.cpd(4, max_iters=50, tol=1e-5, precision="bf16", init=Ud, graph=True)
    h = F.cpd(4, max_iters=50, tol=1e-5, precision="bf16", init=Ud, graph=False)
    f32 = F.cpd(4, max_iters=50, tol=1e-5, precision="fp32", init=Ud)
    assert g["graph"] and not h["graph"]
    assert g["converged"] and f32["converged"]
    assert abs(g["fit"] - fit_o) <= 1e-4, (g["fit"], fit_o)
    assert abs(f32["fit"] - fit_o) <= 1e-4, (f32["fit"], fit_o)
    assert g["iters"] == h["iters"]
    assert abs(g["fit"] - h["fit"]) <= 1e-6


def test_cpd_errors(torch_cuda):
    import mmcsf
    dims = [10, 12, 14]
    X, _, _ = _tensor(dims, 300, seed=1)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF)
    with pytest.raises(mmcsf.MmcsfError):
        F.cpd(12)
    B = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF)
    with pytest.raises(mmcsf.MmcsfError):
        B.cpd(8)


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-4), ("fp64solve", 1e-6)])
def test_cpd_4d_tracks_fp64_oracle(precision, tol, torch_cuda):
    """CP-ALS on a 4-D tensor (the reference's cpd is 3-D only)."""
    import mmcsf
    dims = [30, 25, 20, 15]
    X, inds, vals = _tensor(dims, 6000, seed=44, planted=3, noise=0.01)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=1)
    U, Ud = _init(torch_cuda, dims, 8, seed=45)
    res = F.cpd(8, max_iters=6, tol=1e-12, precision=precision, init=Ud)
    _, lam_o, fit_o, hist_o = CO.cp_als(dims, inds, vals, U, max_iters=6, tol=1e-12)
    assert res["iters"] == 6
    assert np.max(np.abs(np.array(res["history"]) - np.array(hist_o))) <= tol, (res["history"], hist_o)


def test_cpd_resume_from_checkpoint(torch_cuda):
    """Checkpoint/resume: the normalised factors and lambda of a run, with
    lambda folded back into one factor, restart ALS where it stopped; 3 + 3
    iterations give the fits of the 4th..6th iterations of one 6-iteration
    run (the model's scale split does not change an ALS update)."""
    import mmcsf
    torch = torch_cuda
    dims = [40, 55, 30]
    X, _, _ = _tensor(dims, 6000, seed=7, planted=4, noise=0.01)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=1)
    _, Ud = _init(torch, dims, 8, seed=8)
    full = F.cpd(8, max_iters=6, tol=1e-12, precision="fp64solve", init=Ud)
    first = F.cpd(8, max_iters=3, tol=1e-12, precision="fp64solve", init=Ud)
    ck = [f.clone() for f in first["factors"]]
    ck[0] = ck[0] * torch.tensor(first["lambda"], dtype=torch.float32, device="cuda")
    second = F.cpd(8, max_iters=3, tol=1e-12, precision="fp64solve", init=ck)
    assert np.max(np.abs(np.array(second["history"]) - np.array(full["history"][3:]))) <= 1e-6


@pytest.mark.parametrize("precision", ["fp32", "fp64solve", "bf16"])
def test_cpd_graph_matches_host_driven(precision, torch_cuda):
    import mmcsf
    torch = torch_cuda
    dims = [60, 45, 50]
    X, _, _ = _tensor(dims, 8000, seed=21, planted=4, noise=0.01)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=1)
    _, Ud = _init(torch, dims, 8, seed=22)
    g = F.cpd(8, max_iters=12, tol=1e-5, precision=precision, init=Ud, graph=True)
    h = F.cpd(8, max_iters=12, tol=1e-5, precision=precision, init=Ud, graph=False)
    assert g["graph"] and not h["graph"]
    assert g["iters"] == h["iters"] and g["converged"] == h["converged"]
    assert np.max(np.abs(np.array(g["history"]) - np.array(h["history"]))) <= 1e-6, (g["history"], h["history"])
    for a, b in zip(g["factors"], h["factors"]):
        assert torch.allclose(a, b, rtol=1e-4, atol=1e-6)
    if precision != "bf16":  # the default stream cannot be captured: the FP32 forms run host-driven there
        d = F.cpd(8, max_iters=12, tol=1e-5, precision=precision, init=Ud, graph=True,
                  stream=torch.cuda.default_stream())
        assert not d["graph"] and d["iters"] == h["iters"]
        assert np.max(np.abs(np.array(d["history"]) - np.array(h["history"]))) <= 1e-6
