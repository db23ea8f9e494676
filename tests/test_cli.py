"""The `mttkrp` command (mm-csf_b200/bin/mttkrp), which keeps the reference's
flags (-i -m -R -t -f -w -b -v -c -o -h; src/util.h:3341-3442), adds -P (the
partition rule), and keeps its
"Total GPU time ... nSlc/nFibers/nnz" line (src/mttkrp_gpu.cu:3760-3767).

CPU: argument errors end with a message and a nonzero status (the reference
exit(0)s) before any GPU work. GPU: every format and mode, with the
reference's constant factors (U[m] = m + 0.5), checked by the command's own
-c 1 comparison and by its -o output against the FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "mm-csf_b200", "bin", "mttkrp")


def _run(args, timeout=300):
    return subprocess.run([BIN] + args, capture_output=True, text=True, timeout=timeout)


def test_cli_argument_errors(tmp_path):
    assert os.path.exists(BIN), "build mm-csf_b200 first"
    p = _run([])
    assert p.returncode != 0 and "-t implementation type" in p.stdout
    p = _run(["-i", "x.tns", "-t", "7"])
    assert p.returncode != 0 and "-t 7 is not provided" in p.stderr
    p = _run(["-i", "x.tns", "-z", "3"])
    assert p.returncode != 0 and "unknown option" in p.stderr
    p = _run(["-i", str(tmp_path / "missing.tns"), "-t", "12"])
    assert p.returncode != 0 and "load_tensor failed" in p.stderr


@pytest.mark.parametrize("nd", [3, 4])
def test_cli_coo_cpu(nd, tmp_path):
    """-t 1 (the reference's COO CPU path, src/mttkrp.cu:105-109) served by the
    library's host COO MTTKRP: its timing line, and -o equal to the oracle's
    MTTKRP_COO_CPU on the reference's constant factors, which (as in the
    reference) adds to U[mode] = mode + 0.5 without zeroing it."""
    rng = np.random.default_rng(20 + nd)
    dims = [30, 40, 20] if nd == 3 else [12, 10, 9, 8]
    n = 2000
    lin = rng.choice(int(np.prod(dims)), size=n, replace=False)
    inds = [np.asarray(i, np.uint64) for i in np.unravel_index(lin, dims)]
    vals = np.round(rng.random(n) + 0.1, 3).astype(np.float32)
    tns = tmp_path / "x.tns"
    O.write_tns(str(tns), dims, inds, vals)
    R = 8
    U = [np.full((d, R), m + 0.5, np.float32) for m, d in enumerate(dims)]
    for m in range(nd):
        out = tmp_path / f"c_{m}.txt"
        p = _run(["-i", str(tns), "-m", str(m), "-R", str(R), "-t", "1", "-o", str(out)])
        assert p.returncode == 0, p.stderr
        assert "COO CPU - time:" in p.stdout
        head, got = _read_out(out)
        assert head[0] == str(dims[m]) and got.shape == (dims[m], R)
        want = O.mttkrp_coo_f32(inds, vals, m, U) + np.float32(m + 0.5)
        assert np.all(np.abs(got - want) <= 0.006), m  # -o prints %.2f


def _read_out(path):
    with open(path) as fh:
        head = fh.readline().split()
        rows = [[float(v) for v in line.split()] for line in fh if line.strip()]
    return head, np.array(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("nd", [3, 4])
def test_cli_formats_and_modes(nd, tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(nd)
    dims = [50, 70, 40] if nd == 3 else [30, 25, 20, 15]
    n = 4000
    lin = rng.choice(int(np.prod(dims)), size=n, replace=False)
    inds = [np.asarray(i, np.uint64) for i in np.unravel_index(lin, dims)]
    vals = np.round(rng.random(n) + 0.1, 3).astype(np.float32)
    tns = tmp_path / "x.tns"
    O.write_tns(str(tns), dims, inds, vals)  # the reference's .tns: order and lengths, then 1-based entries
    R = 16
    U = [np.full((d, R), m + 0.5, np.float32) for m, d in enumerate(dims)]
    for t, modes in ((12, [0]), (8, range(nd)), (10, range(nd))):
        for m in modes:
            extras = [[], ["-w", "2", "-f", "3"], ["-w", "4"]]
            if t == 12:  # the partition heuristic deciding (-P 1), with -h
                extras += [["-P", "1"], ["-P", "1", "-h", "2", "-f", "3"]]
            for extra in extras:
                out = tmp_path / f"o_{t}_{m}.txt"
                p = _run(["-i", str(tns), "-m", str(m), "-R", str(R), "-t", str(t), "-c", "1", "-o", str(out)]
                         + extra)
                assert p.returncode == 0, (t, m, extra, p.stderr)
                assert "Total GPU time:" in p.stdout and f"nnz:{n}" in p.stdout, p.stdout
                assert "Correctness pass!" in p.stdout, (t, m, extra, p.stdout)
                head, got = _read_out(out)
                assert head[0] == str(dims[m]) and got.shape == (dims[m], R)
                want = O.mttkrp_coo_f64(dims, inds, vals, m, U)
                assert np.all(np.abs(got - want) <= 0.006 + 1e-5 * np.abs(want)), (t, m, extra)
    # the same tensor from a binary COO file
    import mmcsf
    bpath = tmp_path / "x.bin"
    mmcsf.CooTensor.load_tns(str(tns)).write_bin(str(bpath))
    out = tmp_path / "o_bin.txt"
    p = _run(["-i", str(bpath), "-m", "1", "-R", str(R), "-t", "8", "-w", "2", "-c", "1", "-o", str(out)])
    assert p.returncode == 0 and "Correctness pass!" in p.stdout, p.stderr
    _, got = _read_out(out)
    want = O.mttkrp_coo_f64(dims, inds, vals, 1, U)
    assert np.all(np.abs(got - want) <= 0.006 + 1e-5 * np.abs(want))


TTM_BIN = os.path.join(ROOT, "mm-csf_b200", "bin", "ttm")


def test_ttm_cli_argument_errors():
    assert os.path.exists(TTM_BIN), "build mm-csf_b200 first"
    p = subprocess.run([TTM_BIN], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "usage" in p.stdout
    p = subprocess.run([TTM_BIN, "-i", "x.tns", "-t", "1"], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "-t 1 is not provided" in p.stderr


@pytest.mark.gpu
def test_ttm_cli(tmp_path):
    """The ttm command: every mode, with and without a fiber split, against the
    oracle's TTM with the reference's constant factor (leaf mode + 0.5)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(11)
    dims = [50, 70, 40]
    n = 4000
    lin = rng.choice(int(np.prod(dims)), size=n, replace=False)
    inds = [np.asarray(i, np.uint64) for i in np.unravel_index(lin, dims)]
    vals = np.round(rng.random(n) + 0.1, 3).astype(np.float32)
    tns = tmp_path / "x.tns"
    O.write_tns(str(tns), dims, inds, vals)
    for m in range(3):
        for f in (0, 3):
            out = tmp_path / f"y_{m}_{f}.txt"
            args = [TTM_BIN, "-i", str(tns), "-m", str(m), "-R", "16", "-c", "1", "-o", str(out)]
            if f:
                args += ["-f", str(f)]
            p = subprocess.run(args, capture_output=True, text=True, timeout=300)
            assert p.returncode == 0 and "TTM GPU - time" in p.stdout and "Correctness pass!" in p.stdout, p
            head, got = _read_out(out)
            leaf = O.order_modes(dims, m)[2]
            want, _, _ = O.ttm_f32(dims, inds, vals, m, np.full((dims[leaf], 16), leaf + 0.5, np.float32),
                                   f or O.INF_TH)
            assert got.shape == want.shape and np.all(np.abs(got - want) <= 0.006 + 1e-5 * np.abs(want))
