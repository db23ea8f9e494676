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
