"""Test infrastructure, not product code: Python driver for the C oracle.

Restates, step for step, the sequence the reference's `mttkrp` main runs to
build each format (src/mttkrp.cu:72-389), using the C primitives in
oracle/mmcsf_oracle.c, and returns every array under the same names the
reference harness (oracle/ref_harness.cpp) dumps, so the two can be compared
key by key. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg may import this module, and only as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(HERE, "_build")
_LIB_PATH = os.path.join(_BUILD, "libmmcsf_oracle.so")
_REF_LIB = os.path.join(HERE, "_ref", "libmmcsf_ref.so")
_REF_LIB_HEUR = os.path.join(HERE, "_ref", "libmmcsf_ref_heur.so")
INF_TH = 99999999  # the reference's default -f (src/util.h:212)
FBRS_TH_MMCSF = 128  # 4-D fbrS split for -t 12 (src/util.h:1325-1326)
FBRS_TH_OFF = 999999999

_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build(force=False):
    """Compile the C restatement into oracle/_build/libmmcsf_oracle.so."""
    os.makedirs(_BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, "mmcsf_oracle.c"), os.path.join(HERE, "generate.c")]
    if force or not os.path.exists(_LIB_PATH) or any(os.path.getmtime(_LIB_PATH) < os.path.getmtime(s)
                                                     for s in srcs):
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", "-o", _LIB_PATH]
                       + srcs + ["-lm"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def _ptr_array(arrs, ctype=ctypes.c_uint64):
    P = ctypes.POINTER(ctype)
    return (P * len(arrs))(*[a.ctypes.data_as(P) for a in arrs])


# --------------------------------------------------------------------------
# .tns text format: src/util.h:313-370 (load_tensor)
# --------------------------------------------------------------------------
def load_tns(path):
    """Parse a .tns file: line 1 = order, line 2 = dims, then 1-based
    coordinates and a value per line. Returns (dims, inds[nd] uint64 0-based,
    vals float32). The count is the number of parsed entries; the reference
    uses (#lines - 2), which agrees for files without trailing blank lines."""
    with open(path) as fh:
        toks = fh.read().split()
    nd = int(toks[0])
    dims = [int(t) for t in toks[1:1 + nd]]
    body = toks[1 + nd:]
    n = len(body) // (nd + 1)
    a = np.array(body[:n * (nd + 1)], dtype=object).reshape(n, nd + 1) if n else np.zeros((0, nd + 1))
    inds = [np.array(a[:, m], dtype=np.float64).astype(np.uint64) - 1 if n else np.zeros(0, np.uint64)
            for m in range(nd)]
    vals = np.array(a[:, nd], dtype=np.float32) if n else np.zeros(0, np.float32)
    return dims, [np.ascontiguousarray(i, dtype=np.uint64) for i in inds], vals


def write_tns(path, dims, inds, vals):
    """Write a .tns file (1-based coordinates) readable by the reference."""
    nd = len(dims)
    with open(path, "w") as fh:
        fh.write(f"{nd}\n" + " ".join(str(d) for d in dims) + "\n")
        cols = [np.asarray(i, dtype=np.uint64) + 1 for i in inds]
        for x in range(len(vals)):
            fh.write(" ".join(str(int(c[x])) for c in cols) + " " + repr(float(vals[x])) + "\n")


# --------------------------------------------------------------------------
# primitives
# --------------------------------------------------------------------------
def order_modes(dims, mode, natural=False):
    nd = len(dims)
    d = (ctypes.c_uint64 * nd)(*dims)
    out = (ctypes.c_int * nd)()
    lib().orc_order_modes(nd, d, mode, int(natural), out)
    return list(out)


def redundant_mode(orders):
    """src/mttkrp.cu:314-343: the last mode whose (slice, fiber) pair repeats
    an earlier mode's pair swapped; -1 when there is none."""
    redun = -1
    for m in range(1, len(orders)):
        if any(orders[m][1] == orders[p][0] and orders[m][0] == orders[p][1] for p in range(m)):
            redun = m
    return redun


def sort_coo(inds, vals, keys):
    """Stable in-place sort on the key prefix (src/util.h:389-527)."""
    nd = len(inds)
    n = len(vals)
    k = (ctypes.c_int * len(keys))(*keys)
    rc = lib().orc_sort_coo(nd, ctypes.c_uint64(n), _ptr_array(inds),
                            vals.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), k, len(keys))
    assert rc == 0


def create_csf(inds, order, fbr_th, fbrs_th):
    """src/util.h:1320-1436 / 760-850. Returns (ptr[l], idx[l]) lists."""
    nd = len(inds)
    n = len(inds[0])
    L = nd - 1
    ptr = [np.zeros(n + 2, np.uint64) for _ in range(L)]
    idx = [np.zeros(n + 2, np.uint64) for _ in range(L)]
    nptr = (ctypes.c_uint64 * L)()
    nidx = (ctypes.c_uint64 * L)()
    o = (ctypes.c_int * nd)(*order)
    lib().orc_create_csf(nd, ctypes.c_uint64(n), _ptr_array(inds), o, ctypes.c_uint64(fbr_th),
                         ctypes.c_uint64(fbrs_th), _ptr_array(ptr), _ptr_array(idx), nptr, nidx)
    return [ptr[l][:nptr[l]].copy() for l in range(L)], [idx[l][:nidx[l]].copy() for l in range(L)]


def fbr_like_slc(ptr0, idx0):
    nslc = len(idx0)
    nf = int(ptr0[-1]) if len(ptr0) else 0
    out = np.zeros(max(nf, 1), np.uint64)
    lib().orc_fbr_like_slc(ptr0.ctypes.data_as(_u64p), idx0.ctypes.data_as(_u64p),
                           ctypes.c_uint64(nslc), out.ctypes.data_as(_u64p))
    return out[:nf]


def _bins(fn, nd, ptr, tot_nnz):
    nslc = len(ptr[0]) - 1
    bin_of = np.zeros(max(nslc, 1), np.int32)
    fn(nd, _ptr_array(ptr), ctypes.c_uint64(max(nslc, 0)), ctypes.c_uint64(tot_nnz),
       bin_of.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    bin_of = bin_of[:nslc]
    return [np.nonzero(bin_of == b)[0].astype(np.uint64) for b in range(10)]


def keys_per_sort(nd):
    """3-D sorts compare two keys, 4-D sorts three (src/util.h:389-410)."""
    return 2 if nd == 3 else 3


def _csf_dict(pfx, order, ptr, idx, inds, vals, with_fbr_like=True):
    d = {f"{pfx}.nnz": np.array([len(vals)], np.uint64), f"{pfx}.modeOrder": np.array(order, np.uint64)}
    for l in range(len(ptr)):
        d[f"{pfx}.fbrPtr{l}"] = ptr[l]
        d[f"{pfx}.fbrIdx{l}"] = idx[l]
    nfib = len(ptr[1]) if len(ptr) > 1 else 0
    d[f"{pfx}.nFibers"] = np.array([nfib], np.uint64)
    if with_fbr_like:
        d[f"{pfx}.fbrLikeSlcInds"] = fbr_like_slc(ptr[0], idx[0])[:max(nfib - 1, 0)]
    for m in range(len(inds)):
        d[f"{pfx}.inds{m}"] = inds[m].copy()
    d[f"{pfx}.vals"] = vals.copy()
    return d


# --------------------------------------------------------------------------
# format builders (mirror the reference main's call sequence)
# --------------------------------------------------------------------------
def mm_partition(dims, inds_x, orders, xorder, redun, fbth=1):
    """The partition heuristic of mm_partition_reuseBased (src/util.h:2167-2516)
    without its closing `mode = 2;` override (:2517), nonzeros in X's order
    (inds_x: X's arrays after the chain of per-mode sorts). Returns the
    partition of every nonzero (int32)."""
    nd = len(dims)
    n = len(inds_x[0])
    part = np.zeros(max(n, 1), np.int32)
    o = ((ctypes.c_int * 8) * nd)()
    for m in range(nd):
        for i in range(nd):
            o[m][i] = orders[m][i]
    d = (ctypes.c_uint64 * nd)(*dims)
    xo = (ctypes.c_int * nd)(*xorder)
    arrs = [np.ascontiguousarray(i, dtype=np.uint64) for i in inds_x]
    rc = lib().orc_mm_partition(nd, ctypes.c_uint64(n), _ptr_array(arrs), d, o, xo, redun, int(fbth),
                                part.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise ValueError(f"the reference reads out of bounds on this input (code {rc})")
    return part[:n]


def build_mmcsf(dims, inds, vals, mode=0, fbr_th=INF_TH, partition="all-to-last", fbth=1):
    """mttkrp -t 12: src/mttkrp.cu:72-389. partition="all-to-last" is the
    reference as shipped (src/util.h:2517 assigns every nonzero to partition
    2); partition="heuristic" keeps the heuristic's choice (mm_partition,
    with -h = fbth) and fills every partition the way populate_paritions and
    sort_MI_CSF do (src/util.h:2088-2126, 412-527). Returns a dict keyed like
    the reference harness dump."""
    nd = len(dims)
    K = keys_per_sort(nd)
    inds = [np.array(i, dtype=np.uint64) for i in inds]
    vals = np.array(vals, dtype=np.float32)
    xorder = order_modes(dims, mode)
    sort_coo(inds, vals, xorder[:K])
    orders = []
    redun = -1
    for m in range(nd):
        orders.append(order_modes(dims, m))
        if m >= 1 and any(orders[m][1] == orders[p][0] and orders[m][0] == orders[p][1] for p in range(m)):
            redun = m
        if m != redun:
            sort_coo(inds, vals, orders[m][:K])
    if partition == "all-to-last":
        part_of = np.full(len(vals), 2, np.int32)
    elif partition == "heuristic":
        part_of = mm_partition(dims, inds, orders, xorder, redun, fbth)
    else:
        raise NotImplementedError(partition)
    out = {"redunMode": np.array([redun], np.int64), "X.modeOrder": np.array(xorder, np.uint64)}
    for p in range(nd):
        pfx = f"part{p}"
        sel = part_of == p
        if not sel.any():
            out[f"{pfx}.nnz"] = np.array([0], np.uint64)
            out[f"{pfx}.modeOrder"] = np.array(orders[p], np.uint64)
            continue
        pin = [i[sel].copy() for i in inds]
        pv = vals[sel].copy()
        sort_coo(pin, pv, orders[p][:K])
        ptr, idx = create_csf(pin, orders[p], fbr_th, FBRS_TH_MMCSF)
        out.update(_csf_dict(pfx, orders[p], ptr, idx, pin, pv))
    return out


def build_bcsf(dims, inds, vals, mode=0, fbr_th=INF_TH):
    """mttkrp -t 8: src/mttkrp.cu:72-100, 167-236 (create_HCSR, make_KTiling,
    create_TiledHCSR, make_TiledBin, create_fbrLikeSlcInds)."""
    nd = len(dims)
    K = keys_per_sort(nd)
    inds = [np.array(i, dtype=np.uint64) for i in inds]
    vals = np.array(vals, dtype=np.float32)
    order = order_modes(dims, mode)
    sort_coo(inds, vals, order[:K])
    ptr, idx = create_csf(inds, order, fbr_th, FBRS_TH_OFF)
    out = _csf_dict("bcsf", order, ptr, idx, inds, vals)
    for b, sl in enumerate(_bins(lib().orc_tiled_bins, nd, ptr, len(vals))):
        out[f"bcsf.bin{b}"] = sl
    return out


def build_hyb(dims, inds, vals, mode=0, fbr_th=INF_TH):
    """mttkrp -t 10: src/mttkrp.cu:138-151 (create_HCSR, create_HYB[_4D],
    make_HybBin)."""
    nd = len(dims)
    K = keys_per_sort(nd)
    inds = [np.array(i, dtype=np.uint64) for i in inds]
    vals = np.array(vals, dtype=np.float32)
    order = order_modes(dims, mode)
    sort_coo(inds, vals, order[:K])
    ptr, idx = create_csf(inds, order, fbr_th, FBRS_TH_OFF)
    n = len(vals)
    cap = n + 2
    coo = [np.zeros(cap, np.uint64) for _ in range(nd)]
    coov = np.zeros(cap, np.float32)
    cslp, csli, csl1, csl2 = (np.zeros(cap, np.uint64) for _ in range(4))
    cslv = np.zeros(cap, np.float32)
    hptr = [np.zeros(cap, np.uint64) for _ in range(3)]
    hidx = [np.zeros(cap, np.uint64) for _ in range(3)]
    hleaf = np.zeros(cap, np.uint64)
    hv = np.zeros(cap, np.float32)
    counts = np.zeros(10, np.uint64)
    nidx = np.array([len(i) for i in idx], np.uint64)
    fp = ctypes.POINTER(ctypes.c_float)
    o = (ctypes.c_int * nd)(*order)
    lib().orc_create_hyb(nd, ctypes.c_uint64(n), _ptr_array(inds), vals.ctypes.data_as(fp), o,
                         _ptr_array(ptr), _ptr_array(idx), nidx.ctypes.data_as(_u64p), _ptr_array(coo),
                         coov.ctypes.data_as(fp), cslp.ctypes.data_as(_u64p), csli.ctypes.data_as(_u64p),
                         csl1.ctypes.data_as(_u64p), csl2.ctypes.data_as(_u64p), cslv.ctypes.data_as(fp),
                         _ptr_array(hptr), _ptr_array(hidx), hleaf.ctypes.data_as(_u64p),
                         hv.ctypes.data_as(fp), counts.ctypes.data_as(_u64p))
    ncoo, ncsl, nh, ncslslc = (int(c) for c in counts[:4])
    out = {"hyb.COOnnz": np.array([ncoo], np.uint64), "hyb.CSLnnz": np.array([ncsl], np.uint64),
           "hyb.HCSRnnz": np.array([nh], np.uint64), "hyb.modeOrder": np.array(order, np.uint64)}
    for m in range(nd):
        out[f"hyb.COOinds{m}"] = coo[m][:ncoo]
    out["hyb.COOvals"] = coov[:ncoo]
    hp = [hptr[l][:int(counts[4 + l])] for l in range(nd - 1)]
    if nd == 3:
        out["hyb.CSLslicePtr"] = cslp[:ncslslc + 1]
        out["hyb.CSLsliceIdx"] = csli[:ncslslc]
        out["hyb.CSLinds1"] = csl1[:ncsl]
        out["hyb.CSLinds2"] = csl2[:ncsl]
        out["hyb.CSLvals"] = cslv[:ncsl]
    for l in range(nd - 1):
        out[f"hyb.fbrPtr{l}"] = hp[l]
        out[f"hyb.fbrIdx{l}"] = hidx[l][:int(counts[7 + l])]
    out["hyb.indsLeaf"] = hleaf[:nh]
    out["hyb.vals"] = hv[:nh]
    for b, sl in enumerate(_bins(lib().orc_hyb_bins, nd, hp, n)):
        out[f"hyb.bin{b}"] = sl
    if nd == 3:
        cslcnt = np.diff(cslp[:ncslslc + 1].astype(np.int64))
        TB = 512
        LB = [0, 2, 4, 8, 16, 1024, 4 * TB, 8 * TB, 16 * TB, 32 * TB]
        UB = [1025, 5, 9, 17, 1025, 4 * TB + 1, 8 * TB + 1, 16 * TB + 1, 32 * TB + 1, n + 1]
        cb = np.full(ncslslc, -1)
        for s in range(ncslslc):
            for b in range(10):
                if LB[b] < cslcnt[s] < UB[b]:
                    cb[s] = b
                    break
        for b in range(10):
            out[f"hyb.cslbin{b}"] = np.nonzero(cb == b)[0].astype(np.uint64)
    return out


# --------------------------------------------------------------------------
# MTTKRP
# --------------------------------------------------------------------------
def ttm_f32(dims, inds, vals, mode, factor_leaf, fbr_th=INF_TH):
    """TTM_CPU (src/ttm_cpu.cpp:60-86) on the CSF of `mode` as the reference's
    ttm builds it (the sort of mttkrp -t 8, create_HCSR with the -f split).
    Returns (Y (F x R float32, one row per real fiber), ptr, idx) with the
    CSF's pointer and index arrays."""
    order = order_modes(dims, mode)
    sinds = [np.array(i, dtype=np.uint64) for i in inds]
    svals = np.array(vals, dtype=np.float32)
    sort_coo(sinds, svals, order[:2])
    ptr, idx = create_csf(sinds, order, fbr_th, FBRS_TH_OFF)
    F = len(ptr[1]) - 1
    R = factor_leaf.shape[1]
    y = np.zeros((max(F, 1), R), np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    fptr = np.ascontiguousarray(ptr[1], np.uint64)
    leaf = np.ascontiguousarray(sinds[order[2]], np.uint64)
    u = np.ascontiguousarray(factor_leaf, np.float32)
    v = np.ascontiguousarray(svals, np.float32)
    lib().orc_ttm_f32(ctypes.c_uint64(F), fptr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                      leaf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), v.ctypes.data_as(fp),
                      u.ctypes.data_as(fp), R, y.ctypes.data_as(fp))
    return y[:F], ptr, idx


def mttkrp_coo_f32(inds, vals, mode, factors):
    """MTTKRP_COO_CPU semantics (src/mttkrp_cpu.cpp:60-113) with the output
    zeroed first. factors: list of float32 (dim, R) arrays (not modified)."""
    nd = len(inds)
    R = factors[0].shape[1]
    U = [np.ascontiguousarray(f, dtype=np.float32).copy() for f in factors]
    U[mode][:] = 0
    fp = ctypes.POINTER(ctypes.c_float)
    ind = [np.ascontiguousarray(i, dtype=np.uint64) for i in inds]
    v = np.ascontiguousarray(vals, dtype=np.float32)
    lib().orc_mttkrp_coo_f32(nd, ctypes.c_uint64(len(v)), _ptr_array(ind), v.ctypes.data_as(fp), mode, R,
                             (fp * nd)(*[u.ctypes.data_as(fp) for u in U]))
    return U[mode]


def mttkrp_coo_f64(dims, inds, vals, mode, factors):
    """FP64-accumulated MTTKRP: the precision oracle."""
    nd = len(inds)
    R = factors[0].shape[1]
    U = [np.ascontiguousarray(f, dtype=np.float32) for f in factors]
    out = np.zeros((dims[mode], R), np.float64)
    fp = ctypes.POINTER(ctypes.c_float)
    ind = [np.ascontiguousarray(i, dtype=np.uint64) for i in inds]
    v = np.ascontiguousarray(vals, dtype=np.float32)
    d = (ctypes.c_uint64 * nd)(*dims)
    lib().orc_mttkrp_coo_f64(nd, ctypes.c_uint64(len(v)), _ptr_array(ind), v.ctypes.data_as(fp), mode, R,
                             (fp * nd)(*[u.ctypes.data_as(fp) for u in U]), d,
                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


# --------------------------------------------------------------------------
# the reference itself (oracle/_ref), when it was built here
# --------------------------------------------------------------------------
def ref_available():
    return os.path.exists(_REF_LIB)


_ref = None


def ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(_REF_LIB)
    return _ref


def parse_dump(path):
    d = {}
    with open(path) as fh:
        for line in fh:
            t = line.split()
            if not t:
                continue
            name, n = t[0], int(t[1])
            vals = t[2:2 + n]
            if name.endswith("vals") or name.endswith("Vals"):
                d[name] = np.array(vals, dtype=np.float64).astype(np.float32)
            elif name == "redunMode":
                d[name] = np.array(vals, dtype=np.int64)
            else:
                d[name] = np.array(vals, dtype=np.uint64)
    return d


_ref_heur = None


def ref_heur_available():
    return os.path.exists(_REF_LIB_HEUR)


def ref_heur_lib():
    """The reference built without its partition override (oracle/_ref), on
    one OpenMP thread."""
    global _ref_heur
    if _ref_heur is None:
        _ref_heur = ctypes.CDLL(_REF_LIB_HEUR)
        _ref_heur.ref_set_threads(1)
    return _ref_heur


def ref_dump_heuristic(tns_path, mode, fbr_th, mifbth, out_path):
    """The reference's MM-CSF builder with the partition heuristic deciding
    (-h = mifbth)."""
    rc = ref_heur_lib().ref_mmcsf_dump_h(tns_path.encode(), int(mode), ctypes.c_long(int(fbr_th)),
                                         ctypes.c_long(int(mifbth)), out_path.encode())
    if rc != 0:
        raise RuntimeError("ref_mmcsf_dump_h failed")
    return parse_dump(out_path)


def ref_dump(kind, tns_path, mode, fbr_th, out_path):
    """Run the reference's own builder for `kind` in {"mmcsf","bcsf","hyb"}."""
    fn = {"mmcsf": "ref_mmcsf_dump", "bcsf": "ref_bcsf_dump", "hyb": "ref_hyb_dump"}[kind]
    rc = getattr(ref_lib(), fn)(tns_path.encode(), int(mode), ctypes.c_long(int(fbr_th)), out_path.encode())
    if rc != 0:
        raise RuntimeError(f"{fn} failed")
    return parse_dump(out_path)


def ref_ttm(tns_path, mode, fbr_th, factor_leaf, max_fibers):
    """The reference's own TTM_CPU (oracle/_ref) on a .tns file: (Y, F)."""
    R = factor_leaf.shape[1]
    y = np.zeros((max_fibers, R), np.float32)
    n = ctypes.c_uint64()
    fp = ctypes.POINTER(ctypes.c_float)
    u = np.ascontiguousarray(factor_leaf, np.float32)
    rc = ref_lib().ref_ttm(tns_path.encode(), mode, ctypes.c_long(fbr_th), R, u.ctypes.data_as(fp),
                           y.ctypes.data_as(fp), ctypes.c_uint64(max_fibers), ctypes.byref(n))
    assert rc == 0, "fiber capacity too small"
    return y[:n.value], int(n.value)


def ref_mttkrp_coo(dims, inds, vals, mode, factors):
    """The reference's MTTKRP_COO_CPU on these arrays, output zeroed first."""
    nd = len(dims)
    R = factors[0].shape[1]
    U = [np.ascontiguousarray(f, dtype=np.float32).copy() for f in factors]
    U[mode][:] = 0
    fp = ctypes.POINTER(ctypes.c_float)
    ind = [np.ascontiguousarray(i, dtype=np.uint64) for i in inds]
    v = np.ascontiguousarray(vals, dtype=np.float32)
    d = (ctypes.c_uint64 * nd)(*dims)
    rc = ref_lib().ref_coo_mttkrp(nd, d, ctypes.c_uint64(len(v)), _ptr_array(ind), v.ctypes.data_as(fp),
                                  mode, R, (fp * nd)(*[u.ctypes.data_as(fp) for u in U]))
    assert rc == 0
    return U[mode]


# --------------------------------------------------------------------------
# Seeded synthetic tensors on the host: oracle/generate.c restates the
# library's generator (mmcsf_generate) for the benchmark's CPU legs.
# --------------------------------------------------------------------------
def generate(dims, nnz, dist, zipf_s=1.0, val_dist=0, seed=0, threads=0):
    """(inds[nd] uint32, vals float32) of the seeded tensor mmcsf_generate
    makes for the same arguments (uniform / Zipf modes; values uniform (0,1],
    lognormal or integers 1..50), computed on `threads` host threads."""
    nd = len(dims)
    d = (ctypes.c_uint64 * 4)(*[int(x) for x in dims] + [0] * (4 - nd))
    ds = (ctypes.c_int * 4)(*[int(x) for x in (dist if isinstance(dist, (list, tuple)) else [dist] * nd)]
                            + [0] * (4 - nd))
    zs = (ctypes.c_double * 4)(*[float(x) for x in (zipf_s if isinstance(zipf_s, (list, tuple)) else [zipf_s] * nd)]
                               + [0.0] * (4 - nd))
    inds = [np.empty(int(nnz), np.uint32) for _ in range(nd)]
    vals = np.empty(int(nnz), np.float32)
    T = threads or len(os.sched_getaffinity(0))
    u32p = ctypes.POINTER(ctypes.c_uint32)
    rc = lib().orc_generate(nd, d, ctypes.c_uint64(int(nnz)), ds, zs, int(val_dist), ctypes.c_uint64(int(seed)),
                            int(T), (u32p * nd)(*[i.ctypes.data_as(u32p) for i in inds]),
                            vals.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    if rc != 0:
        raise RuntimeError(f"orc_generate failed ({rc})")
    return inds, vals


# --------------------------------------------------------------------------
# The reference's own GPU MTTKRP (src/mttkrp_gpu.cu:3380-3784), built for
# sm_100a as oracle/_ref/libmmcsf_ref_gpu.so by oracle/build_ref.py.
# --------------------------------------------------------------------------
_REF_GPU_LIB = os.path.join(HERE, "_ref", "libmmcsf_ref_gpu.so")
_ref_gpu = None


def ref_gpu_available():
    return os.path.exists(_REF_GPU_LIB)


def ref_gpu_lib():
    global _ref_gpu
    if _ref_gpu is None:
        _ref_gpu = ctypes.CDLL(_REF_GPU_LIB)
    return _ref_gpu


def ref_mihcsr_gpu(dims, R, part, mode_order, fbr_ptr, fbr_idx, fbr_like, leaf, vals, warp_per_slice=4,
                   tb_size=128, fiber_per_warp=1):
    """Run MTTKRP_MIHCSR_GPU on one MM-CSF partition given by the reference's
    arrays (fbr_ptr / fbr_idx per level, fbrLikeSlcInds, the leaf index of
    every nonzero, values), with the reference's constant factors U[m] = m +
    0.5 and its -w / -b / -s. Returns (Total GPU time in ms as it prints it, the
    last mode's output)."""
    nd = len(dims)
    u64 = ctypes.c_uint64
    P = ctypes.POINTER(u64)
    fp = [np.ascontiguousarray(a, dtype=np.uint64) for a in fbr_ptr]
    fi = [np.ascontiguousarray(a, dtype=np.uint64) for a in fbr_idx]
    nfib = len(fp[-1])
    like = np.ascontiguousarray(fbr_like, dtype=np.uint64)
    if len(like) < nfib:  # the reference's copy reads nFibers entries; the last one it leaves unset
        like = np.concatenate([like, np.full(nfib - len(like), like[-1] if len(like) else 0, np.uint64)])
    lf = np.ascontiguousarray(leaf, dtype=np.uint64)
    v = np.ascontiguousarray(vals, dtype=np.float32)
    out = np.zeros((dims[-1], R), np.float32)
    ms = ctypes.c_double()
    rc = ref_gpu_lib().ref_mihcsr_gpu(
        nd, (u64 * nd)(*[int(d) for d in dims]), int(R), int(warp_per_slice), int(tb_size), int(fiber_per_warp),
        int(part),
        (ctypes.c_int * nd)(*[int(m) for m in mode_order]), (P * (nd - 1))(*[a.ctypes.data_as(P) for a in fp]),
        (u64 * (nd - 1))(*[len(a) for a in fp]), (P * (nd - 1))(*[a.ctypes.data_as(P) for a in fi]),
        (u64 * (nd - 1))(*[len(a) for a in fi]), like.ctypes.data_as(P), u64(nfib),
        (P * nd)(*[lf.ctypes.data_as(P)] * nd), v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), u64(len(v)),
        out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_mihcsr_gpu failed ({rc})")
    return ms.value, out
