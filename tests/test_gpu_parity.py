"""Parity of the CUDA path (through the C ABI) with the reference.

* format arrays: bit-exact against the reference's own builders (golden
  fixtures) and against the C oracle on fresh random tensors;
* MTTKRP: within 1e-5 relative (Frobenius, and per element against
  |ref| + 1e-6 * max|ref|) of the FP64 oracle, for every mode and many ranks;
* full-size runs: size-independent properties (column checksums in FP64).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-5


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _rand_coo(rng, dims, n, skew=False, dup=False):
    if skew:
        inds = [np.minimum(rng.zipf(1.4, n) - 1, d - 1).astype(np.uint64) for d in dims]
    else:
        inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    if not dup:
        key = np.zeros(n, np.uint64)
        for m, d in enumerate(dims):
            key = key * np.uint64(d) + inds[m]
        _, first = np.unique(key, return_index=True)
        first = np.sort(first)
        inds = [i[first] for i in inds]
    vals = (rng.random(len(inds[0])) + 0.05).astype(np.float32)
    return inds, vals


def _sentinel_key(kind, nd):
    pfx = {"mmcsf": "part2", "bcsf": "bcsf", "hyb": "hyb"}[kind]
    if kind == "hyb":  # create_HYB pushes no sentinel
        return pfx, None, None
    return pfx, f"{pfx}.fbrIdx{nd - 2}", f"{pfx}.fbrPtr{nd - 2}"


def _compare_dumps(ref, got, kind, nd, ctx):
    pfx, skey, pkey = _sentinel_key(kind, nd)
    for k, v in ref.items():
        assert k in got, (ctx, k)
        g = got[k]
        if k.endswith("vals"):
            assert np.array_equal(np.asarray(v, np.float32), g), (ctx, k)
            continue
        v = np.asarray(v).astype(np.int64)
        g = np.asarray(g).astype(np.int64)
        if k == skey and len(v):
            # The reference's sentinel is read one past the last nonzero when
            # the last fiber holds 2+ nonzeros; it is only defined otherwise.
            ptr = np.asarray(ref[pkey], np.int64)
            defined = len(ptr) < 2 or ptr[-1] - ptr[-2] == 1 or int(ref[f"{pfx}.nnz"][0]) == 1
            assert len(v) == len(g), (ctx, k)
            assert np.array_equal(v[:-1], g[:-1]), (ctx, k)
            if defined:
                assert v[-1] == g[-1], (ctx, k, "sentinel")
            continue
        assert len(v) == len(g) and np.array_equal(v, g), (ctx, k, v[:12], g[:12])


def _check_close(got, ref64, ctx):
    got = np.asarray(got, np.float64)
    scale = np.abs(ref64).max() if ref64.size else 0.0
    fro = np.linalg.norm(got - ref64) / max(np.linalg.norm(ref64), 1e-30)
    assert fro <= RTOL, (ctx, "frobenius", fro)
    if ref64.size:
        rel = np.abs(got - ref64) / (np.abs(ref64) + 1e-6 * scale + 1e-30)
        assert rel.max() <= RTOL * 10, (ctx, "max rel", rel.max())


def test_golden_format_arrays_bit_exact(golden_cases, torch_cuda):
    import mmcsf
    n = 0
    for case in golden_cases:
        dims = case["dims"]
        X = mmcsf.CooTensor.from_arrays(dims, case["inds"], case["vals"])
        for fmt in case["formats"]:
            impl = {"mmcsf": mmcsf.IMPL_MMCSF, "bcsf": mmcsf.IMPL_BCSF, "hyb": mmcsf.IMPL_HBCSF}[fmt["kind"]]
            F = mmcsf.Format(X, impl=impl, mode=fmt["mode"], fiber_threshold=fmt["f"], keep_coo=True)
            _compare_dumps(fmt["arrays"], F.reference_dump(), fmt["kind"], len(dims),
                           (case["name"], fmt["kind"], fmt["mode"], fmt["f"]))
            n += 1
    assert n >= 60


def test_golden_mttkrp(golden_cases, torch_cuda):
    import mmcsf
    torch = torch_cuda
    for case in golden_cases:
        dims = case["dims"]
        X = mmcsf.CooTensor.from_arrays(dims, case["inds"], case["vals"])
        inds = [np.array(i, np.uint64) for i in case["inds"]]
        vals = np.array(case["vals"], np.float32)
        U = [np.array(u, np.float32).reshape(d, -1) for u, d in zip(case["factors"], dims)]
        Ud = [torch.tensor(u, device="cuda") for u in U]
        F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=2)
        outs = F.mttkrp_all(Ud)
        torch.cuda.synchronize()
        for mt in case["mttkrp"]:
            m = mt["mode"]
            ref32 = np.array(mt["out"], np.float32).reshape(dims[m], -1)
            ref64 = O.mttkrp_coo_f64(dims, inds, vals, m, U)
            got = outs[m].cpu().numpy()
            _check_close(got, ref64, (case["name"], m))
            # the reference's own FP32 output agrees to the same tolerance
            assert np.linalg.norm(ref32 - ref64) / max(np.linalg.norm(ref64), 1e-30) <= RTOL
        for m in range(len(dims)):  # single-mode B-CSF and HB-CSF
            for impl in (mmcsf.IMPL_BCSF, mmcsf.IMPL_HBCSF):
                B = mmcsf.Format(X, impl=impl, mode=m, fiber_threshold=3)
                got = B.mttkrp(m, Ud).cpu().numpy()
                _check_close(got, O.mttkrp_coo_f64(dims, inds, vals, m, U), (case["name"], impl, m))


CASES = [
    # nd, dims, nnz, skew, dup, f
    (3, [300, 500, 200], 20000, False, False, 0),
    (3, [300, 500, 200], 20000, True, False, 16),
    (3, [64, 2000, 40], 30000, True, False, 1),
    (3, [50, 50, 50], 8000, False, True, 5),
    (4, [200, 40, 30, 10], 30000, False, False, 0),
    (4, [300, 20, 10, 6], 30000, True, False, 3),
    (4, [5, 3, 4, 2000], 20000, False, False, 0),  # long (o0,o1) runs: fbrS split at 128
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_random_formats_match_oracle(case, torch_cuda):
    import mmcsf
    nd, dims, n, skew, dup, f = CASES[case]
    rng = np.random.default_rng(100 + case)
    inds, vals = _rand_coo(rng, dims, n, skew, dup)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    fth = f if f else O.INF_TH
    for mode in range(nd):
        ref = O.build_mmcsf(dims, inds, vals, mode, fth)
        F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=mode, fiber_threshold=f, keep_coo=True)
        _compare_dumps(ref, F.reference_dump(), "mmcsf", nd, ("mmcsf", case, mode))
        refb = O.build_bcsf(dims, inds, vals, mode, fth)
        B = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=mode, fiber_threshold=f, keep_coo=True)
        _compare_dumps(refb, B.reference_dump(), "bcsf", nd, ("bcsf", case, mode))
        refh = O.build_hyb(dims, inds, vals, mode, fth)
        Hf = mmcsf.Format(X, impl=mmcsf.IMPL_HBCSF, mode=mode, fiber_threshold=f)
        _compare_dumps(refh, Hf.reference_dump(), "hyb", nd, ("hyb", case, mode))


@pytest.mark.parametrize("R", [1, 4, 8, 12, 16, 32, 48, 64, 128, 256])
def test_mttkrp_all_modes_any_rank(R, torch_cuda):
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(R)
    for nd, dims, n, skew in ((3, [120, 300, 80], 15000, True), (4, [60, 30, 20, 40], 15000, False)):
        inds, vals = _rand_coo(rng, dims, n, skew)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        Ud = [torch.tensor(u, device="cuda") for u in U]
        for f in (0, 7):
            F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f)
            outs = F.mttkrp_all(Ud)
            torch.cuda.synchronize()
            for m in range(nd):
                _check_close(outs[m].cpu().numpy(), O.mttkrp_coo_f64(dims, inds, vals, m, U), (nd, R, f, m))


@pytest.mark.parametrize("chunk", [1, 3, 32, 100, 4096])
def test_chunk_sizes(chunk, torch_cuda):
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(chunk)
    dims = [40, 90, 30]
    inds, vals = _rand_coo(rng, dims, 6000, True)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    U = [rng.random((d, 32)).astype(np.float32) for d in dims]
    Ud = [torch.tensor(u, device="cuda") for u in U]
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=0)
    outs = F.mttkrp_all(Ud, cfg={"chunk": chunk})
    torch.cuda.synchronize()
    for m in range(3):
        _check_close(outs[m].cpu().numpy(), O.mttkrp_coo_f64(dims, inds, vals, m, U), (chunk, m))


def test_generator_distinct_deterministic(torch_cuda):
    import mmcsf
    dims = [2000, 3000, 50]
    a = mmcsf.CooTensor.generate(dims, 200000, dist=[1, 1, 1], zipf_s=1.1, val_dist=mmcsf.VAL_LOGNORMAL, seed=3)
    b = mmcsf.CooTensor.generate(dims, 200000, dist=[1, 1, 1], zipf_s=1.1, val_dist=mmcsf.VAL_LOGNORMAL, seed=3)
    ia, va = a.host_arrays()
    ib, vb = b.host_arrays()
    for m in range(3):
        assert np.array_equal(ia[m], ib[m])
        assert ia[m].max() < dims[m]
    assert np.array_equal(va, vb)
    key = (ia[0].astype(np.uint64) * 3000 + ia[1]) * 50 + ia[2]
    assert len(np.unique(key)) == len(key) == 200000
    assert (va > 0).all()
    # skew: the hottest slice of a Zipf(1.1) mode holds far more than the mean
    cnt = np.bincount(ia[2], minlength=50)
    assert cnt.max() > 3 * cnt.mean()


def test_mttkrp_host_entry_point(torch_cuda):
    import mmcsf
    rng = np.random.default_rng(9)
    dims = [100, 80, 60]
    inds, vals = _rand_coo(rng, dims, 5000)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    U = [rng.random((d, 32)).astype(np.float32) for d in dims]
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF)
    for _ in range(2):
        outs = F.mttkrp_all_host(U)
        for m in range(3):
            _check_close(outs[m], O.mttkrp_coo_f64(dims, inds, vals, m, U), ("host", m))


def test_errors_are_status_codes(torch_cuda):
    import mmcsf
    torch = torch_cuda
    dims = [10, 10, 10]
    X = mmcsf.CooTensor.from_arrays(dims, [np.array([1]), np.array([2]), np.array([3])], np.array([1.0]))
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.Format(X, impl=7)
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=3)
    B = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=1)
    U = [torch.rand(10, 8, device="cuda") for _ in range(3)]
    with pytest.raises(mmcsf.MmcsfError):
        B.mttkrp(0, U)  # built for mode 1 only
    with pytest.raises(mmcsf.MmcsfError):
        B.mttkrp_all(U)


def _fp64_mttkrp_dev(torch, inds, vals, U, mode, chunk=4_000_000):
    """FP64 MTTKRP on the device from the COO nonzeros (the checker for
    tensors too large for the host oracle)."""
    R = U[0].shape[1]
    out = torch.zeros(U[mode].shape[0], R, dtype=torch.float64, device="cuda")
    U64 = [u.double() for u in U]
    for s_ in range(0, vals.numel(), chunk):
        t = vals[s_:s_ + chunk].double()[:, None].repeat(1, R)
        for q in range(len(U)):
            if q != mode:
                t = t * U64[q][inds[q][s_:s_ + chunk].long()]
        out.index_add_(0, inds[mode][s_:s_ + chunk].long(), t)
    return out


def _check_close_dev(torch, got, ref, ctx):
    d = got.double() - ref
    fro = float(d.norm() / ref.norm())
    scale = float(ref.abs().max())
    rel = float((d.abs() / (ref.abs() + 1e-6 * scale)).max())
    assert fro <= RTOL and rel <= RTOL * 10, (ctx, fro, rel)


@pytest.mark.parametrize("views", [1, 0])
def test_full_size_skewed_elementwise(views, torch_cuda):
    """500k x 2M x 20k-shaped Zipf(1.1) tensor at 20M nonzeros, every mode
    element by element against an FP64 MTTKRP (default and tuned plans).
    With views=0 the leaf mode scatters one reduction per nonzero, as the
    reference's kernel does (src/mttkrp_gpu.cu:1438-1472); its hottest rows
    receive ~10^6 terms, accumulated in FP64, so it meets 1e-5 like every
    other traversal."""
    import mmcsf
    torch = torch_cuda
    dims = [500000, 2000000, 20000]
    X = mmcsf.CooTensor.generate(dims, 20_000_000, dist=[1, 1, 1], zipf_s=1.1, val_dist=mmcsf.VAL_LOGNORMAL,
                                 seed=11)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=0, views=views)
    g = torch.Generator(device="cuda").manual_seed(0)
    U = [torch.rand(d, 32, device="cuda", generator=g) for d in dims]
    di, dv = X.device_tensors()
    refs = [_fp64_mttkrp_dev(torch, di, dv, U, m) for m in range(3)]
    outs = F.mttkrp_all(U)
    for m in range(3):
        _check_close_dev(torch, outs[m], refs[m], ("default", views, m))
    F.tune(U)
    for rep in range(2):
        outs = F.mttkrp_all(U)
        for m in range(3):
            _check_close_dev(torch, outs[m], refs[m], ("tuned", views, m, rep))


@pytest.mark.parametrize("R", [4, 32, 128, 256])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_kernel_variants_3d(R, dtype, torch_cuda):
    """The 3-D kernels (per-team fiber walk, branch-free fiber walk,
    per-nonzero walk, per-nonzero walk with the middle row once per fiber,
    vector index loads, warp-interleaved walk, rows staged in shared memory) at
    every occupancy level, on the partition and on the views, with fiber
    splits and with many short slices (slice changes inside most blocks)."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(300 + R)
    cases = (([150, 400, 60], 20000, True), ([3000, 50, 40], 9000, False))
    for dims, n, skew in cases:
        inds, vals = _rand_coo(rng, dims, n, skew)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        if dtype == "bf16":
            Ud = [torch.tensor(u, device="cuda").to(torch.bfloat16) for u in U]
            U = [t.float().cpu().numpy() for t in Ud]
        else:
            Ud = [torch.tensor(u, device="cuda") for u in U]
        ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(3)]
        for f in (0, 3):
            F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f, views=2)
            for m in range(3):
                travs = (1, 2) if F.info(4 + m)["present"] else (1,)
                for trav in travs:
                    for kern in (1, 2, 3, 4, 5, 6, 7):
                        for mb in (1, 2, 3, 4):
                            for chunk in (64, 1000):
                                cfg = {"traversal": trav, "kernel": kern, "min_blocks": mb, "chunk": chunk}
                                out = F.mttkrp(m, Ud, cfg=cfg)
                                _check_close(out.cpu().numpy(), ref[m], (dims, f, m, cfg))
            if f == 0:
                B = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=1, fiber_threshold=4)
                for kern in (1, 2, 3, 4, 5, 6, 7):
                    out = B.mttkrp(1, Ud, cfg={"kernel": kern})
                    _check_close(out.cpu().numpy(), ref[1], ("bcsf", dims, kern))


@pytest.mark.parametrize("R", [4, 32, 128])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_kernel_variants_4d(R, dtype, torch_cuda):
    """4-D: the per-team fiber walk and the per-nonzero walk at every occupancy
    level, on the partition (fbrS split at 128) and on every mode's view."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(400 + R)
    for dims, n, skew in (([40, 30, 50, 20], 20000, True), ([900, 8, 6, 5], 6000, False)):
        inds, vals = _rand_coo(rng, dims, n, skew)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        if dtype == "bf16":
            Ud = [torch.tensor(u, device="cuda").to(torch.bfloat16) for u in U]
            U = [t.float().cpu().numpy() for t in Ud]
        else:
            Ud = [torch.tensor(u, device="cuda") for u in U]
        ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(4)]
        for f in (0, 3):
            F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f, views=2)
            for m in range(4):
                travs = (1, 2) if F.info(4 + m)["present"] else (1,)
                for trav in travs:
                    for kern in (1, 3):
                        for mb in (1, 2, 3, 4):
                            for chunk in (64, 1000):
                                cfg = {"traversal": trav, "kernel": kern, "min_blocks": mb, "chunk": chunk}
                                out = F.mttkrp(m, Ud, cfg=cfg)
                                _check_close(out.cpu().numpy(), ref[m], (dims, f, m, cfg))


@pytest.mark.parametrize("R", [16, 32, 64, 128])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_staged_walk_edges(R, dtype, torch_cuda):
    """Kernel 7 (rows staged in shared memory, even nonzero ranges per team):
    nonzero counts below, at and just past a team's 8-nonzero step and a
    block's share (most teams empty, ranges ending mid-step), one slice, one
    fiber, fibers of one nonzero, a middle index repeated across slices, at
    every stage count, single mode and two-output walk, against the FP64
    oracle."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(700 + R)
    cases = [([4, 5, 6], 1), ([4, 5, 6], 7), ([4, 5, 6], 9), ([9, 9, 9], 300), ([1, 30, 4000], 3000),
             ([1, 1, 5000], 4000), ([5000, 3, 1], 2500), ([60, 2, 300], 20000), ([3000, 40, 3000], 50000)]
    for dims, n in cases:
        inds, vals = _rand_coo(rng, dims, n)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        if dtype == "bf16":
            Ud = [torch.tensor(u, device="cuda").to(torch.bfloat16) for u in U]
            U = [t.float().cpu().numpy() for t in Ud]
        else:
            Ud = [torch.tensor(u, device="cuda") for u in U]
        ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(3)]
        for f in (0, 2):
            F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f, views=2)
            m0, m1 = F.pair_modes()
            for mb in (1, 2, 3, 4):
                for m in range(3):
                    for trav in ((1, 2) if F.info(4 + m)["present"] else (1,)):
                        cfg = {"traversal": trav, "kernel": 7, "min_blocks": mb}
                        _check_close(F.mttkrp(m, Ud, cfg=cfg).cpu().numpy(), ref[m], (dims, n, f, m, cfg))
                for rep in range(2):  # the outputs are zeroed by every call
                    outs = F.mttkrp_pair(Ud, cfg={"kernel": 7, "min_blocks": mb})
                    for m in (m0, m1):
                        _check_close(outs[m].cpu().numpy(), ref[m], ("pair", dims, n, f, mb, m, rep))


@pytest.mark.parametrize("R", [4, 8, 32, 64, 128])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_two_output_walk(R, dtype, torch_cuda):
    """mmcsf_mttkrp_pair: the partition's slice and middle modes from one walk
    match the FP64 oracle at every occupancy level and chunk, with fiber
    splits, with many short slices, and through mttkrp_all / the host-buffer
    call once a plan selects it."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(500 + R)
    cases = (([150, 400, 60], 20000, True), ([3000, 50, 40], 9000, False), ([5, 7, 900], 3000, False))
    for dims, n, skew in cases:
        inds, vals = _rand_coo(rng, dims, n, skew)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        if dtype == "bf16":
            Ud = [torch.tensor(u, device="cuda").to(torch.bfloat16) for u in U]
            U = [t.float().cpu().numpy() for t in Ud]
        else:
            Ud = [torch.tensor(u, device="cuda") for u in U]
        ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(3)]
        for f in (0, 3):
            F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f, views=1)
            m0, m1 = F.pair_modes()
            order = F.info(2)["mode_order"]
            assert (m0, m1) == (order[0], order[1])
            for kern in (2, 3, 4, 5, 6, 7):
                for mb in (1, 2, 3, 4):
                    for chunk in (1, 32, 100, 1024):
                        outs = F.mttkrp_pair(Ud, cfg={"min_blocks": mb, "chunk": chunk, "kernel": kern})
                        assert set(outs) == {m0, m1}
                        for m in (m0, m1):
                            _check_close(outs[m].cpu().numpy(), ref[m], (dims, f, m, kern, mb, chunk))
            plan = F.tune(Ud)
            plan["pair"].update(use=False)
            F.set_plan(plan)
            F.mttkrp_all(Ud)
            separate = F.last_launches
            for kern in (2, 3, 4, 5, 6, 7):
                plan["pair"].update(use=True, chunk=256, min_blocks=2, kernel=kern)
                F.set_plan(plan)
                for _ in range(2):
                    outs = F.mttkrp_all(Ud)
                    assert F.last_launches == separate - 1
                    for m in range(3):
                        _check_close(outs[m].cpu().numpy(), ref[m], ("all+pair", dims, f, kern, m))
            if dtype == "f32":
                houts = F.mttkrp_all_host(U)
                for m in range(3):
                    _check_close(houts[m], ref[m], ("host+pair", dims, f, m))
            # a caller's traversal or kernel override turns the walk off
            outs = F.mttkrp_all(Ud, cfg={"kernel": 1})
            assert F.last_launches == separate
            for m in range(3):
                _check_close(outs[m].cpu().numpy(), ref[m], ("override", dims, f, m))


@pytest.mark.parametrize("R", [4, 32, 128])
@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_two_output_walk_4d(R, dtype, torch_cuda):
    """The 4-D two-output walk (slice mode and level-1 mode of the partition)
    against the FP64 oracle: every launch shape and chunk, fiber splits, the
    fbrS split at 128 (long (o0, o1) runs), and through the all-mode calls."""
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(600 + R)
    cases = (([40, 30, 50, 20], 20000, True), ([900, 8, 6, 5], 6000, False), ([5, 3, 4, 2000], 20000, False))
    for dims, n, skew in cases:
        inds, vals = _rand_coo(rng, dims, n, skew)
        X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        if dtype == "bf16":
            Ud = [torch.tensor(u, device="cuda").to(torch.bfloat16) for u in U]
            U = [t.float().cpu().numpy() for t in Ud]
        else:
            Ud = [torch.tensor(u, device="cuda") for u in U]
        ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(4)]
        for f in (0, 3):
            F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f, views=2)
            m0, m1 = F.pair_modes()
            assert (m0, m1) == tuple(F.info(2)["mode_order"][:2])
            for mb in (1, 2, 3, 4):
                for chunk in (1, 32, 100, 1024):
                    outs = F.mttkrp_pair(Ud, cfg={"min_blocks": mb, "chunk": chunk})
                    for m in (m0, m1):
                        _check_close(outs[m].cpu().numpy(), ref[m], (dims, f, m, mb, chunk))
            plan = F.tune(Ud)
            plan["pair"].update(use=True, chunk=512, min_blocks=2, kernel=3)
            F.set_plan(plan)
            outs = F.mttkrp_all(Ud)
            for m in range(4):
                _check_close(outs[m].cpu().numpy(), ref[m], ("all+pair", dims, f, m))
            if dtype == "f32":
                houts = F.mttkrp_all_host(U)
                for m in range(4):
                    _check_close(houts[m], ref[m], ("host+pair", dims, f, m))


def test_two_output_walk_errors(torch_cuda):
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(77)
    dims = [20, 30, 10, 8]
    inds, vals = _rand_coo(rng, dims, 2000)
    U = [torch.rand(d, 16, device="cuda") for d in dims]
    X3 = mmcsf.CooTensor.from_arrays(dims[:3], inds[:3], vals)
    B = mmcsf.Format(X3, impl=mmcsf.IMPL_BCSF, mode=0)
    with pytest.raises(mmcsf.MmcsfError):
        B.mttkrp_pair(U[:3])
    F = mmcsf.Format(X3, impl=mmcsf.IMPL_MMCSF)
    with pytest.raises(mmcsf.MmcsfError):
        F.mttkrp_pair([torch.rand(d, 256, device="cuda") for d in dims[:3]])  # R above 128
    with pytest.raises(mmcsf.MmcsfError):
        F.set_plan({"pair": {"use": True, "chunk": -1, "min_blocks": 1}})
    with pytest.raises(mmcsf.MmcsfError):
        F.set_plan({"pair": {"use": True, "chunk": 256, "min_blocks": 1, "kernel": 8}})


@pytest.mark.parametrize("nd", [3, 4])
def test_views_and_tuner(nd, torch_cuda):
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(40 + nd)
    dims = [150, 400, 60] if nd == 3 else [80, 50, 30, 40]
    inds, vals = _rand_coo(rng, dims, 20000, True)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    U = [rng.random((d, 32)).astype(np.float32) for d in dims]
    Ud = [torch.tensor(u, device="cuda") for u in U]
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, views=2)
    order = F.info(2)["mode_order"]
    ref = [O.mttkrp_coo_f64(dims, inds, vals, m, U) for m in range(nd)]
    for m in range(nd):
        v = F.info(4 + m)
        assert v["present"] == (m != order[0]) and (not v["present"] or v["mode_order"][0] == m)
        for trav in (1, 2):
            if trav == 2 and not v["present"]:
                with pytest.raises(mmcsf.MmcsfError):
                    F.mttkrp(m, Ud, cfg={"traversal": 2})
                continue
            out = F.mttkrp(m, Ud, cfg={"traversal": trav})
            _check_close(out.cpu().numpy(), ref[m], ("view", nd, m, trav))
    plan = F.tune(Ud)
    assert set(plan) == set(range(nd)) | {"pair", "dtype", "mixed", "fiber_threshold"}
    assert plan["dtype"] == "f32" and plan["mixed"] is False
    assert plan["pair"]["use"] in (True, False) and (nd == 3 or not plan["pair"]["use"])
    outs = F.mttkrp_all(Ud)
    torch.cuda.synchronize()
    for m in range(nd):
        _check_close(outs[m].cpu().numpy(), ref[m], ("tuned", nd, m))
    # views=1 builds only the leaf-level mode's view
    F1 = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, views=1)
    present = [F1.info(4 + m)["present"] for m in range(nd)]
    assert present == [m == order[-1] for m in range(nd)]


@pytest.mark.parametrize("nd", [3, 4])
def test_hbcsf_mttkrp_random(nd, torch_cuda):
    import mmcsf
    torch = torch_cuda
    rng = np.random.default_rng(70 + nd)
    dims = [3000, 40, 30] if nd == 3 else [2000, 20, 15, 10]
    inds, vals = _rand_coo(rng, dims, 20000, True)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    for R in (16, 32, 24):
        U = [rng.random((d, R)).astype(np.float32) for d in dims]
        Ud = [torch.tensor(u, device="cuda") for u in U]
        for mode in range(nd):
            for f in (0, 1, 2):
                H = mmcsf.Format(X, impl=mmcsf.IMPL_HBCSF, mode=mode, fiber_threshold=f)
                ref = O.mttkrp_coo_f64(dims, inds, vals, mode, U)
                for kern in (0, 1, 3):  # default, per-team walk, per-nonzero walk on the CSF part
                    got = H.mttkrp(mode, Ud, cfg={"kernel": kern} if kern else None).cpu().numpy()
                    _check_close(got, ref, ("hyb", nd, R, mode, f, kern))
