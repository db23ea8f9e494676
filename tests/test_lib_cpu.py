"""Host-side checks that need no GPU: the C-ABI library loads, exports every
entry point include/mmcsf.h declares, and its host code (the .tns parser and
argument validation) agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    with open(os.path.join(ROOT, "include", "mmcsf.h")) as fh:
        src = fh.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(mmcsf_[a-z0-9_]+)\s*\(", src, re.M):
        names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from mmcsf import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, f"binding missing for {n}"
    # the bounds-checked build exports the same interface
    B = ctypes.CDLL(os.path.join(ROOT, "mm-csf_b200", "lib", "libmmcsf_bounds.so"))
    for n in sorted(names):
        assert hasattr(B, n), ("bounds build", n)


def test_status_strings_and_version():
    from mmcsf import _lib
    L = _lib.lib()
    assert L.mmcsf_status_string(0) == b"ok"
    assert L.mmcsf_status_string(1) == b"invalid argument"
    assert L.mmcsf_version() >= 100


def test_tns_loader_matches_oracle(golden_cases, tmp_path):
    import mmcsf
    for case in golden_cases:
        p = str(tmp_path / (case["name"] + ".tns"))
        dims = case["dims"]
        inds = [np.array(i, np.uint64) for i in case["inds"]]
        vals = np.array(case["vals"], np.float32)
        O.write_tns(p, dims, inds, vals)
        X = mmcsf.CooTensor.load_tns(p)
        nd, d2, nnz = X.info()
        assert d2 == dims and nnz == len(vals)
        gi, gv = X.host_arrays()
        for m in range(nd):
            assert np.array_equal(gi[m].astype(np.uint64), inds[m])
        assert np.array_equal(gv, vals)


def test_loader_errors_are_status_codes(tmp_path):
    import mmcsf
    with pytest.raises(mmcsf.MmcsfError) as e:
        mmcsf.CooTensor.load_tns(str(tmp_path / "missing.tns"))
    assert e.value.status == 4
    bad = tmp_path / "bad.tns"
    bad.write_text("5\n2 2 2 2 2\n1 1 1 1 1 1.0\n")
    with pytest.raises(mmcsf.MmcsfError) as e:
        mmcsf.CooTensor.load_tns(str(bad))
    assert e.value.status == 1
    oob = tmp_path / "oob.tns"
    oob.write_text("3\n2 2 2\n1 3 1 1.0\n")
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.CooTensor.load_tns(str(oob))


def test_from_arrays_validates_indices():
    import mmcsf
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.CooTensor.from_arrays([2, 2, 2], [np.array([0]), np.array([5]), np.array([0])], np.array([1.0]))
    X = mmcsf.CooTensor.from_arrays([2, 3, 4], [np.array([1]), np.array([2]), np.array([3])], np.array([2.5]))
    assert X.info() == (3, [2, 3, 4], 1)


def test_tns_parallel_parse_and_binary_roundtrip(tmp_path):
    """A multi-megabyte .tns (parsed by several host threads) gives exactly the
    oracle's sequential parse; junk ends the entries where a sequential parse
    stops; an out-of-range coordinate is an error; the binary COO file
    round-trips the tensor."""
    import mmcsf
    rng = np.random.default_rng(5)
    dims = [300, 200, 100]
    n = 250000
    inds = [rng.integers(0, d, n).astype(np.uint64) for d in dims]
    vals = (rng.random(n) * 10).astype(np.float32)
    path = str(tmp_path / "big.tns")
    O.write_tns(path, dims, inds, vals)
    X = mmcsf.CooTensor.load_tns(path)
    got_i, got_v = X.host_arrays()
    ref_dims, ref_i, ref_v = O.load_tns(path)
    assert X.dims == [int(d) for d in ref_dims] and X.nnz == len(ref_v) == n
    for a, b in zip(got_i, ref_i):
        assert np.array_equal(a.astype(np.uint64), np.asarray(b, np.uint64))
    assert np.array_equal(got_v.view(np.uint32), np.asarray(ref_v, np.float32).view(np.uint32))
    with open(path, "a") as fh:
        fh.write("1 1 x 0.5\n2 2 2 1.0\n")
    assert mmcsf.CooTensor.load_tns(path).nnz == n
    bad = str(tmp_path / "bad.tns")
    with open(bad, "w") as fh:
        fh.write("3\n2 2 2\n1 1 1 1.0\n1 3 1 2.0\n")
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.CooTensor.load_tns(bad)
    bpath = str(tmp_path / "big.bin")
    X.write_bin(bpath)
    Y = mmcsf.CooTensor.load_bin(bpath)
    yi, yv = Y.host_arrays()
    assert Y.dims == X.dims and Y.nnz == n
    assert all(np.array_equal(a, b) for a, b in zip(yi, got_i)) and np.array_equal(yv, got_v)
    with open(bpath, "r+b") as fh:
        fh.write(b"NOTMAGIC")
    with pytest.raises(mmcsf.MmcsfError):
        mmcsf.CooTensor.load_bin(bpath)


@pytest.mark.parametrize("nd", [3, 4])
def test_host_coo_mttkrp_matches_oracle(nd):
    """-t 1 served by the library (mmcsf_mttkrp_coo_host): one thread is the
    reference's loop bit for bit (through the oracle, itself bit-exact to the
    reference's MTTKRP_COO_CPU); several threads agree within FP32 rounding;
    like the reference it adds to the output it is given."""
    import mmcsf
    rng = np.random.default_rng(7 + nd)
    dims = [40, 33, 27, 5][:nd]
    n = 3000
    inds = [rng.integers(0, d, n).astype(np.uint32) for d in dims]
    vals = rng.random(n).astype(np.float32)
    X = mmcsf.CooTensor.from_arrays(dims, inds, vals)
    R = 12
    U = [rng.random((d, R)).astype(np.float32) for d in dims]
    for mode in range(nd):
        ref = O.mttkrp_coo_f32(inds, vals, mode, U)
        out = np.zeros((dims[mode], R), np.float32)
        X.mttkrp_host(mode, U, out, threads=1)
        assert np.array_equal(out, ref)
        out4 = np.zeros((dims[mode], R), np.float32)
        X.mttkrp_host(mode, U, out4, threads=4)
        assert np.allclose(out4, ref, rtol=1e-5, atol=1e-6)
        base = np.full((dims[mode], R), mode + 0.5, np.float32)
        X.mttkrp_host(mode, U, base, threads=1)
        assert np.allclose(base, ref + (mode + 0.5), rtol=1e-5, atol=1e-5)


def test_host_coo_mttkrp_argument_errors():
    import mmcsf
    X = mmcsf.CooTensor.from_arrays([4, 4, 4], [np.zeros(2, np.uint32)] * 3, np.ones(2, np.float32))
    U = [np.ones((4, 4), np.float32)] * 3
    with pytest.raises(mmcsf.MmcsfError):
        X.mttkrp_host(3, U, np.zeros((4, 4), np.float32))
    with pytest.raises(mmcsf.MmcsfError):
        X.mttkrp_host(0, U, np.zeros((4, 4), np.float64))
