"""The host restatement of the seeded generator (oracle/generate.c), which the
benchmark's CPU legs use so they never load the CUDA library.

CPU: against a sequential Python statement of the same definition (first
`nnz` distinct candidates in candidate order), including tiny coordinate
spaces where duplicates force several rounds, and independent of the thread
count. GPU: bit-identical to the library's mmcsf_generate (indices and
values) for every distribution the benchmark uses."""
import math
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle as O

M64 = (1 << 64) - 1


def _splitmix(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def _u01(h):
    return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0)


def _hash3(seed, stream, j):
    return _splitmix(_splitmix(seed ^ ((stream * 0xD1B54A32D192ED03) & M64)) ^ j)


def _sequential(dims, nnz, dist, s, val_dist, seed):
    nd = len(dims)
    cdf, perm = [], []
    for m, d in enumerate(dims):
        if dist[m] == 1:
            acc, c = 0.0, []
            for k in range(d):
                acc += math.pow(k + 1, -s)
                c.append(acc)
            c = [x / acc for x in c]
            c[-1] = 1.0
            p = list(range(d))
            st = _splitmix(seed ^ (0xABCDEF12345 + m))
            for k in range(d - 1, 0, -1):
                st = _splitmix(st)
                r = st % (k + 1)
                p[k], p[r] = p[r], p[k]
            cdf.append(c)
            perm.append(p)
        else:
            cdf.append(None)
            perm.append(None)

    def coord(m, j):
        u = _u01(_hash3(seed, m + 1, j))
        if dist[m] == 0:
            return min(int(u * dims[m]), dims[m] - 1)
        lo, hi = 0, dims[m] - 1
        while lo < hi:
            mid = (lo + hi) >> 1
            if cdf[m][mid] < u:
                lo = mid + 1
            else:
                hi = mid
        return perm[m][lo]

    seen, kept, j = set(), [], 0
    while len(kept) < nnz:
        c = tuple(coord(m, j) for m in range(nd))
        if c not in seen:
            seen.add(c)
            kept.append((j, c))
        j += 1
    inds = [np.array([c[m] for _, c in kept], np.uint32) for m in range(nd)]
    vals = []
    for jj, _ in kept:
        u1, u2 = _u01(_hash3(seed, 101, jj)), _u01(_hash3(seed, 102, jj))
        if val_dist == 1:
            vals.append(math.exp(math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2)))
        elif val_dist == 2:
            vals.append(1 + int(u1 * 50.0 if u1 * 50.0 < 50.0 else 49.0))
        else:
            # fused multiply-add, rounded once (exact rational arithmetic, then one rounding)
            vals.append(float(Fraction(-u1) * Fraction(1.0 - 1e-7) + 1))
    return inds, np.array(vals, np.float32)


CASES = [  # dims, nnz, dist, s, val, seed
    ([6, 5, 7], 150, [0, 0, 0], 1.0, 0, 3),          # 150 of 210 coordinates: many rounds of duplicates
    ([40, 9, 30], 2000, [1, 1, 1], 1.1, 1, 0),        # Zipf, lognormal
    ([20, 11, 6, 4], 3000, [1, 1, 1, 0], 1.0, 2, 5),  # 4-D, integer values
    ([500, 300, 200], 5000, [1, 0, 1], 1.05, 0, 9),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_host_generator_matches_definition(case):
    dims, nnz, dist, s, val, seed = CASES[case]
    want_i, want_v = _sequential(dims, nnz, dist, s, val, seed)
    for T in (1, 3):
        got_i, got_v = O.generate(dims, nnz, dist, s, val, seed, threads=T)
        for m in range(len(dims)):
            assert np.array_equal(got_i[m], want_i[m]), (case, T, m)
        assert np.array_equal(got_v, want_v), (case, T)


def test_host_generator_thread_independent_large():
    a = O.generate([500000, 2000000, 20000], 300000, [1, 1, 1], 1.1, 1, 0, threads=1)
    b = O.generate([500000, 2000000, 20000], 300000, [1, 1, 1], 1.1, 1, 0, threads=7)
    assert all(np.array_equal(x, y) for x, y in zip(a[0], b[0])) and np.array_equal(a[1], b[1])


GPU_CASES = [  # the benchmark's workloads at reduced nonzero counts, plus a duplicate-heavy space
    ([1000, 1000, 1000], 100000, [0, 0, 0], 1.0, 0, 0),
    ([500000, 2000000, 20000], 2000000, [1, 1, 1], 1.1, 1, 0),
    ([1000000, 20000, 5000, 200], 1400000, [1, 1, 1, 0], 1.0, 2, 0),
    ([100000, 50000, 10000], 500000, [1, 1, 1], 1.05, 0, 13),
    ([6, 5, 7], 150, [0, 0, 0], 1.0, 1, 3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_host_generator_bit_identical_to_device(case):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mmcsf
    dims, nnz, dist, s, val, seed = GPU_CASES[case]
    X = mmcsf.CooTensor.generate(dims, nnz, dist=dist, zipf_s=s, val_dist=val, seed=seed)
    di, dv = X.host_arrays()
    hi, hv = O.generate(dims, nnz, dist, s, val, seed)
    for m in range(len(dims)):
        assert np.array_equal(di[m], hi[m]), (case, m)
    assert np.array_equal(dv.view(np.uint32), hv.view(np.uint32)), (case, int(np.sum(dv != hv)))
