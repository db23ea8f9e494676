"""The reference's own GPU MTTKRP (MTTKRP_MIHCSR_GPU, built for sm_100a from
its sources as oracle/_ref/libmmcsf_ref_gpu.so), driven on the MM-CSF arrays
this library builds (bit-exact to the reference's builders): its last mode's
output matches the FP64 oracle at R <= 32, the ranks its kernels are correct
for (src/mttkrp_gpu.cu:746-753), so the benchmark's reference-GPU timing runs
the reference's kernels on valid data."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("R", [8, 32])
def test_reference_gpu_on_our_arrays(R):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not O.ref_gpu_available():
        pytest.skip("reference GPU library not built (needs the reference sources where build() ran)")
    import mmcsf
    rng = np.random.default_rng(31 + R)
    dims = [300, 800, 60]
    n = 30000
    p = np.arange(1, 801, dtype=np.float64) ** -1.1
    inds = [rng.integers(0, dims[0], n), rng.choice(800, n, p=p / p.sum()), rng.integers(0, dims[2], n)]
    key = (inds[0] * dims[1] + inds[1]) * dims[2] + inds[2]
    _, first = np.unique(key, return_index=True)
    inds = [i[np.sort(first)].astype(np.uint32) for i in inds]
    vals = (rng.random(len(inds[0])) + 0.1).astype(np.float32)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0)
    part = 2
    info = F.info(part)
    order = info["mode_order"]
    ms, out = O.ref_mihcsr_gpu(dims, R, part, order, [F.export(part, "fbrPtr0"), F.export(part, "fbrPtr1")],
                               [F.export(part, "fbrIdx0"), F.export(part, "fbrIdx1")],
                               F.export(part, "fbrLikeSlcInds"), F.export(part, "indsLeaf"),
                               F.export_f32(part, "vals"))
    assert ms > 0
    U = [np.full((d, R), m + 0.5, np.float32) for m, d in enumerate(dims)]
    want = O.mttkrp_coo_f64(dims, [i.astype(np.uint64) for i in inds], vals, 2, U)
    assert np.abs(out - want).max() <= 1e-4 * np.abs(want).max()
