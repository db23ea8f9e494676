"""Python host binding for the B200-native MM-CSF MTTKRP library.

Everything here calls the C ABI in include/mmcsf.h through ctypes; PyTorch is
only used to hold device memory and to name the current CUDA stream. The
reference (isratnisa/MM-CSF) equivalents are noted per call.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import (BuildOpts, CpdOpts, CpdResult, GenSpec, KernelCfg, MmcsfError, PartInfo, Plan, c_f32p, c_u32p, c_u64, c_u64p, c_voidp,
                   check, lib)

IMPL_BCSF = 8
IMPL_HBCSF = 10
IMPL_MMCSF = 12
DTYPE_F32 = 0
DTYPE_BF16 = 1
DIST_UNIFORM = 0
DIST_ZIPF = 1
VAL_UNIFORM01 = 0
VAL_LOGNORMAL = 1
VAL_INT1_50 = 2

__all__ = ["CooTensor", "Format", "autotune", "MmcsfError", "KernelCfg", "IMPL_BCSF", "IMPL_HBCSF", "IMPL_MMCSF",
           "DTYPE_F32", "DTYPE_BF16", "current_stream"]


def current_stream():
    """cudaStream_t of torch's current stream (None when torch has no CUDA)."""
    try:
        import torch
        if torch.cuda.is_available():
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    except ImportError:
        pass
    return None


def _stream(s):
    if s is None:
        return current_stream()
    if isinstance(s, int):
        return ctypes.c_void_p(s)
    if hasattr(s, "cuda_stream"):
        return ctypes.c_void_p(s.cuda_stream)
    return s


class CooTensor:
    """A COO tensor (replaces Tensor + load_tensor, src/util.h:80-104, 313-370)."""

    def __init__(self, handle):
        self._h = handle

    # -- constructors ---------------------------------------------------------
    @classmethod
    def load_tns(cls, path):
        h = c_voidp()
        check(lib().mmcsf_coo_load_tns(path.encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load_bin(cls, path):
        """A binary COO file written by write_bin (no text parse)."""
        h = c_voidp()
        check(lib().mmcsf_coo_load_bin(path.encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, dims, inds, vals):
        nd = len(dims)
        d = (c_u64 * nd)(*[int(x) for x in dims])
        ind = [np.ascontiguousarray(i, dtype=np.uint32) for i in inds]
        v = np.ascontiguousarray(vals, dtype=np.float32)
        ptrs = (c_u32p * nd)(*[i.ctypes.data_as(c_u32p) for i in ind])
        h = c_voidp()
        check(lib().mmcsf_coo_create(nd, d, c_u64(len(v)), ptrs, v.ctypes.data_as(c_f32p), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_device(cls, dims, inds, vals, stream=None):
        """Copy device arrays (torch CUDA tensors: int32/uint32 indices per
        mode, float32 values) into a new handle (mmcsf_coo_create_device)."""
        nd = len(dims)
        d = (c_u64 * nd)(*[int(x) for x in dims])
        ind = [i.contiguous() for i in inds]
        v = vals.contiguous()
        ptrs = (c_voidp * nd)(*[ctypes.c_void_p(i.data_ptr()) for i in ind])
        h = c_voidp()
        check(lib().mmcsf_coo_create_device(nd, d, c_u64(int(v.numel())), ptrs, ctypes.c_void_p(v.data_ptr()),
                                            _stream(stream), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, dims, nnz, dist=DIST_UNIFORM, zipf_s=1.0, val_dist=VAL_UNIFORM01, seed=0, stream=None,
                 planted_rank=0, noise=0.0, poisson=False):
        """Seeded synthetic tensor generated on the device (see mmcsf_generate).
        planted_rank > 0: values from a planted CP model (+ relative Gaussian
        noise, or Poisson counts)."""
        nd = len(dims)
        sp = GenSpec()
        sp.nd = nd
        for m in range(nd):
            sp.dims[m] = int(dims[m])
            sp.dist[m] = dist[m] if isinstance(dist, (list, tuple)) else dist
            sp.zipf_s[m] = zipf_s[m] if isinstance(zipf_s, (list, tuple)) else zipf_s
        sp.nnz = int(nnz)
        sp.val_dist = val_dist
        sp.seed = int(seed)
        sp.planted_rank = int(planted_rank)
        sp.noise = float(noise)
        sp.poisson = 1 if poisson else 0
        h = c_voidp()
        check(lib().mmcsf_generate(ctypes.byref(sp), _stream(stream), ctypes.byref(h)))
        return cls(h)

    # -- queries --------------------------------------------------------------
    def info(self):
        nd = ctypes.c_int()
        dims = (c_u64 * 4)()
        nnz = c_u64()
        check(lib().mmcsf_coo_info(self._h, ctypes.byref(nd), dims, ctypes.byref(nnz)))
        return nd.value, [int(dims[m]) for m in range(nd.value)], int(nnz.value)

    @property
    def nd(self):
        return self.info()[0]

    @property
    def dims(self):
        return self.info()[1]

    @property
    def nnz(self):
        return self.info()[2]

    def host_arrays(self):
        """Copies of (inds[nd] uint32, vals float32) on the host."""
        nd, _, nnz = self.info()
        check(lib().mmcsf_coo_to_host(self._h))
        ip = (c_voidp * 4)()
        vp = c_voidp()
        check(lib().mmcsf_coo_host_arrays(self._h, ip, ctypes.byref(vp)))
        inds = [np.ctypeslib.as_array(ctypes.cast(ip[m], c_u32p), (nnz,)).copy() if nnz else np.zeros(0, np.uint32)
                for m in range(nd)]
        vals = (np.ctypeslib.as_array(ctypes.cast(vp, c_f32p), (nnz,)).copy() if nnz
                else np.zeros(0, np.float32))
        return inds, vals

    def device_tensors(self):
        """Borrowed torch views (int32 indices per mode, float32 values) of the
        device copy; valid while this tensor is alive. Indices must be < 2^31."""
        import torch
        nd, _, nnz = self.info()
        check(lib().mmcsf_coo_to_device(self._h, current_stream()))
        ip = (c_voidp * 4)()
        vp = c_voidp()
        check(lib().mmcsf_coo_device_arrays(self._h, ip, ctypes.byref(vp)))
        inds = [torch.as_tensor(_CudaArray(ip[m], nnz, "<i4"), device="cuda") for m in range(nd)]
        vals = torch.as_tensor(_CudaArray(vp.value, nnz, "<f4"), device="cuda")
        return inds, vals

    def mttkrp_host(self, mode, factors, out, threads=0):
        """-t 1: COO MTTKRP on the host (mmcsf_mttkrp_coo_host; replaces
        MTTKRP_COO_CPU, src/mttkrp_cpu.cpp:60-113). ADDS X_(mode) to `out`
        (numpy float32 dims[mode] x R, C-contiguous) like the reference;
        factors: numpy float32 arrays (the mode's own entry is ignored)."""
        nd, dims, _ = self.info()
        if not 0 <= mode < nd:
            raise MmcsfError(1, "Mode cannot be larger than tensor dimension.")
        check(lib().mmcsf_coo_to_host(self._h))
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.shape[0] != dims[mode]:
            raise MmcsfError(1, "out must be a C-contiguous float32 dims[mode] x R array")
        R = out.shape[1]
        fs = [np.ascontiguousarray(f, dtype=np.float32) for f in factors]
        ptrs = (c_voidp * nd)(*[f.ctypes.data if m != mode else None for m, f in enumerate(fs)])
        check(lib().mmcsf_mttkrp_coo_host(self._h, int(mode), int(R), ptrs, out.ctypes.data, int(threads)))
        return out

    def write_tns(self, path):
        check(lib().mmcsf_coo_write_tns(self._h, path.encode()))

    def write_bin(self, path):
        check(lib().mmcsf_coo_write_bin(self._h, path.encode()))

    def close(self):
        if self._h:
            lib().mmcsf_coo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def _ptr(t):
    """Device pointer of a torch tensor (must be contiguous)."""
    if not t.is_contiguous():
        raise MmcsfError(1, "factor matrices must be contiguous row-major")
    return ctypes.c_void_p(t.data_ptr())


class Format:
    """A device-resident sparse format built from a CooTensor.

    impl follows the reference's -t: 12 = MM-CSF (all modes), 8 = B-CSF,
    10 = HB-CSF (single mode `mode`). fiber_threshold is -f (0 = the
    reference default). partition_rule 0 is the reference as shipped (every
    nonzero in partition 2); 1 lets its partition heuristic decide
    (mm_partition_reuseBased without the override at src/util.h:2517), with
    partition_ratio as -h. views: 0 none, 1 for the modes at the partition's
    leaf level, 2 for every mode (CSFs with the mode at level 0, for MTTKRP);
    view_order 0 orders a view's other modes as the reference orders a
    mode-m CSF (ascending length), 1 longest first (the smallest factor at
    the leaf). Replaces the builder chain the reference's main runs
    (src/mttkrp.cu:72-389)."""

    def __init__(self, coo, impl=IMPL_MMCSF, mode=0, fiber_threshold=0, keep_coo=False, views=0,
                 partition_rule=0, partition_ratio=0, stream=None, view_order=0):
        o = BuildOpts()
        o.impl = impl
        o.mode = mode
        o.fiber_threshold = int(fiber_threshold)
        o.partition_rule = int(partition_rule)
        o.keep_coo = 1 if keep_coo else 0
        o.views = int(views)
        o.partition_ratio = int(partition_ratio)
        o.view_order = int(view_order)
        h = c_voidp()
        check(lib().mmcsf_build(coo._h, ctypes.byref(o), _stream(stream), ctypes.byref(h)))
        self._h = h
        self.impl = impl
        self.mode = mode
        self.nd, self.dims, self.nnz = coo.info()

    def close(self):
        if getattr(self, "_h", None):
            lib().mmcsf_format_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def info(self, part):
        pi = PartInfo()
        check(lib().mmcsf_format_info(self._h, part, ctypes.byref(pi)))
        return {"present": bool(pi.present), "mode_order": [pi.mode_order[i] for i in range(pi.nd)],
                "nnz": int(pi.nnz), "n_slices": int(pi.n_slices), "n_fbrs": int(pi.n_fbrs),
                "n_fibers": int(pi.n_fibers), "device_bytes": int(pi.device_bytes)}

    def check(self, rows=None, stream=None):
        """Validate every index the kernels dereference (mmcsf_format_check):
        index arrays below `rows` (the factors' row counts; default the
        tensor's dims), pointers, fiber flags, per-nonzero indices and chunk
        tables. Raises MmcsfError naming the array and first bad position."""
        r = None
        if rows is not None:
            r = (c_u64 * 4)(*[int(x) for x in rows] + [0] * (4 - len(rows)))
        check(lib().mmcsf_format_check(self._h, r, _stream(stream)))

    def chunk_for_warps(self, warps, R):
        """The worker-team chunk equivalent to the reference's -w `warps`
        warps per fiber (src/util.h:194, src/mttkrp_gpu.cu:3616-3630): the
        reference launches warps*F warps (F fibers over the partitions); the
        kernels here have 32/G teams per warp (G lanes per factor row), so
        the same worker count means max(1, N*G / (32*warps*F)) nonzeros per
        team. The `mttkrp` command maps -w the same way."""
        fibers = sum(self.info(p)["n_fibers"] for p in self.partitions())
        r4 = (int(R) + 3) // 4
        G = 32 if r4 >= 32 else 16 if r4 >= 16 else 8 if r4 >= 8 else 4 if r4 >= 4 else 2 if r4 >= 2 else 1
        return int(max(1, min(1 << 20, self.nnz * G // (32 * int(warps) * max(1, fibers)))))

    def meta(self):
        r = ctypes.c_int()
        xo = (ctypes.c_int * 4)()
        check(lib().mmcsf_format_meta(self._h, ctypes.byref(r), xo))
        return r.value, [xo[i] for i in range(self.nd)]

    def export(self, part, name):
        n = c_u64()
        check(lib().mmcsf_format_export(self._h, part, name.encode(), None, 0, ctypes.byref(n)))
        out = np.zeros(max(int(n.value), 1), np.uint64)
        check(lib().mmcsf_format_export(self._h, part, name.encode(), out.ctypes.data_as(c_u64p), c_u64(len(out)),
                                        ctypes.byref(n)))
        return out[:int(n.value)]

    def export_f32(self, part, name):
        n = c_u64()
        check(lib().mmcsf_format_export_f32(self._h, part, name.encode(), None, 0, ctypes.byref(n)))
        out = np.zeros(max(int(n.value), 1), np.float32)
        check(lib().mmcsf_format_export_f32(self._h, part, name.encode(), out.ctypes.data_as(c_f32p),
                                            c_u64(len(out)), ctypes.byref(n)))
        return out[:int(n.value)]

    def reference_dump(self):
        """Every array under the reference's names (the keys the reference
        harness writes), for bit-exact comparison."""
        d = {}
        nd = self.nd
        if self.impl == IMPL_MMCSF:
            redun, xo = self.meta()
            d["redunMode"] = np.array([redun], np.int64)
            d["X.modeOrder"] = np.array(xo, np.uint64)
            for p in range(nd):
                inf = self.info(p)
                pfx = f"part{p}"
                d[f"{pfx}.nnz"] = np.array([inf["nnz"] if inf["present"] else 0], np.uint64)
                d[f"{pfx}.modeOrder"] = np.array(inf["mode_order"], np.uint64)
                if inf["present"]:
                    self._dump_csf(d, p, pfx, nd)
        elif self.impl == IMPL_BCSF:
            pfx = "bcsf"
            inf = self.info(0)
            d[f"{pfx}.nnz"] = np.array([inf["nnz"]], np.uint64)
            d[f"{pfx}.modeOrder"] = np.array(inf["mode_order"], np.uint64)
            self._dump_csf(d, 0, pfx, nd)
            for b in range(10):
                d[f"{pfx}.bin{b}"] = self.export(0, f"bin{b}")
        else:  # HB-CSF: part 0 = CSF slices, 1 = COO part, 2 = CSL part (3-D)
            inf = self.info(0)
            coo = [self.export(1, f"COOinds{l}") for l in range(nd)]
            d["hyb.COOnnz"] = np.array([len(coo[0])], np.uint64)
            d["hyb.HCSRnnz"] = np.array([inf["nnz"] if inf["present"] else 0], np.uint64)
            d["hyb.modeOrder"] = np.array(inf["mode_order"], np.uint64)
            for l in range(nd):
                d[f"hyb.COOinds{l}"] = coo[l]
            d["hyb.COOvals"] = self.export_f32(1, "COOvals")
            if nd == 3:
                d["hyb.CSLslicePtr"] = self.export(2, "CSLslicePtr")
                d["hyb.CSLsliceIdx"] = self.export(2, "CSLsliceIdx")
                d["hyb.CSLinds1"] = self.export(2, "CSLinds1")
                d["hyb.CSLinds2"] = self.export(2, "CSLinds2")
                d["hyb.CSLvals"] = self.export_f32(2, "CSLvals")
                d["hyb.CSLnnz"] = np.array([len(d["hyb.CSLinds1"])], np.uint64)
                for b in range(10):
                    d[f"hyb.cslbin{b}"] = self.export(2, f"cslbin{b}")
            else:
                d["hyb.CSLnnz"] = np.array([0], np.uint64)
            for l in range(nd - 1):
                d[f"hyb.fbrPtr{l}"] = self.export(0, f"fbrPtr{l}")
                d[f"hyb.fbrIdx{l}"] = self.export(0, f"fbrIdx{l}")
            d["hyb.indsLeaf"] = self.export(0, "indsLeaf")
            d["hyb.vals"] = self.export_f32(0, "vals")
            for b in range(10):
                d[f"hyb.bin{b}"] = self.export(0, f"bin{b}")
        return d

    def _dump_csf(self, d, p, pfx, nd):
        for l in range(nd - 1):
            d[f"{pfx}.fbrPtr{l}"] = self.export(p, f"fbrPtr{l}")
            d[f"{pfx}.fbrIdx{l}"] = self.export(p, f"fbrIdx{l}")
        d[f"{pfx}.nFibers"] = np.array([len(d[f"{pfx}.fbrPtr1"])], np.uint64)
        d[f"{pfx}.fbrLikeSlcInds"] = self.export(p, "fbrLikeSlcInds")
        try:
            for m in range(nd):
                d[f"{pfx}.inds{m}"] = self.export(p, f"inds{m}")
        except MmcsfError:
            pass
        d[f"{pfx}.vals"] = self.export_f32(p, "vals")

    # -- MTTKRP ---------------------------------------------------------------
    def _cfg(self, cfg):
        if cfg is None:
            return None
        if isinstance(cfg, KernelCfg):
            return ctypes.byref(cfg)
        c = KernelCfg()
        for k, v in cfg.items():
            setattr(c, k, v)
        return ctypes.byref(c)

    @staticmethod
    def _dtype(factors):
        import torch
        dt = factors[0].dtype
        if any(f.dtype != dt for f in factors):
            raise MmcsfError(1, "all factors must share one dtype")
        if dt == torch.float32:
            return DTYPE_F32
        if dt == torch.bfloat16:
            return DTYPE_BF16
        raise MmcsfError(1, f"unsupported factor dtype {dt}")

    def mttkrp(self, mode, factors, out=None, cfg=None, stream=None):
        """MTTKRP for one mode; factors: list of CUDA tensors (dims[m] x R,
        float32 or bfloat16). Returns out (dims[mode] x R float32)."""
        import torch
        R = factors[0].shape[1]
        if out is None:
            out = torch.empty((self.dims[mode], R), dtype=torch.float32, device=factors[0].device)
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        check(lib().mmcsf_mttkrp(self._h, mode, R, self._dtype(factors), fp, _ptr(out), self._cfg(cfg),
                                 _stream(stream)))
        return out

    def pair_modes(self):
        """(slice mode, middle mode) of the MM-CSF partition the two-output
        walk runs on; raises MmcsfError when the format has none (4-D, B-CSF)."""
        if getattr(self, "_pair_modes", None) is None:
            modes = (ctypes.c_int * 2)()
            check(lib().mmcsf_mttkrp_pair(self._h, 4, 0, None, None, None, modes, None, None))
            self._pair_modes = (modes[0], modes[1])
        return self._pair_modes

    def mttkrp_pair(self, factors, outs=None, cfg=None, stream=None):
        """The partition's slice and middle modes in one walk
        (mmcsf_mttkrp_pair). Returns {mode: output} for the two modes."""
        import torch
        R = factors[0].shape[1]
        m0, m1 = self.pair_modes()
        modes = None
        if outs is None:
            outs = {m: torch.empty((self.dims[m], R), dtype=torch.float32, device=factors[0].device) for m in (m0, m1)}
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        check(lib().mmcsf_mttkrp_pair(self._h, R, self._dtype(factors), fp, _ptr(outs[m0]), _ptr(outs[m1]), modes,
                                      self._cfg(cfg), _stream(stream)))
        return outs

    def mttkrp_all(self, factors, outs=None, cfg=None, stream=None):
        import torch
        R = factors[0].shape[1]
        if outs is None:
            outs = [torch.empty((d, R), dtype=torch.float32, device=factors[0].device) for d in self.dims]
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        op = (c_voidp * self.nd)(*[_ptr(o) for o in outs])
        check(lib().mmcsf_mttkrp_all(self._h, R, self._dtype(factors), fp, op, self._cfg(cfg), _stream(stream)))
        return outs

    def mttkrp_all_host(self, factors, outs=None, cfg=None, stream=None):
        """All modes through host buffers (numpy float32, ideally pinned)."""
        R = factors[0].shape[1]
        if outs is None:
            outs = [np.empty((d, R), np.float32) for d in self.dims]
        fp = (c_voidp * self.nd)(*[ctypes.c_void_p(_host_ptr(f)) for f in factors])
        op = (c_voidp * self.nd)(*[ctypes.c_void_p(_host_ptr(o)) for o in outs])
        check(lib().mmcsf_mttkrp_all_host(self._h, R, fp, op, self._cfg(cfg), _stream(stream)))
        return outs

    def _plan_dict(self, pl):
        n = self.nd if self.impl == IMPL_MMCSF else 1
        modes = list(range(self.nd)) if self.impl == IMPL_MMCSF else [self.mode]
        dn = {DTYPE_F32: "f32", DTYPE_BF16: "bf16"}
        plan = {m: {"traversal": pl.traversal[m], "chunk": pl.chunk[m], "min_blocks": pl.min_blocks[m],
                    "kernel": pl.kernel[m], "ms": pl.ms[m]} for m in modes[:n]}
        if pl.mixed:
            for m in modes[:n]:
                plan[m].update(dtype=dn[pl.mode_dtype[m]], bf16_error=pl.bf16_error[m], ms_f32=pl.ms_f32[m],
                               ms_bf16=pl.ms_bf16[m])
        if self.impl == IMPL_MMCSF:
            plan["pair"] = {"use": bool(pl.pair), "chunk": pl.pair_chunk, "min_blocks": pl.pair_min_blocks,
                            "kernel": pl.pair_kernel, "ms": pl.pair_ms}
            if pl.mixed:
                plan["pair"].update(dtype=dn[pl.pair_dtype], ms_f32=pl.pair_ms_f32, ms_bf16=pl.pair_ms_bf16)
        plan["dtype"] = dn[pl.factor_dtype]
        plan["mixed"] = bool(pl.mixed)
        plan["fiber_threshold"] = pl.fiber_threshold
        if pl.mixed:
            plan["convert_ms"] = pl.convert_ms
        return plan

    def tune(self, factors, outs=None, stream=None):
        """Autotune traversal, kernel, chunk and occupancy per mode for the
        factors' type (mmcsf_tune; one plan is kept per factor type); returns
        the plan: {mode: {...}} plus, for MM-CSF, "pair": the two-output
        walk's best setting and whether mttkrp_all uses it, and "dtype",
        "fiber_threshold"."""
        import torch
        R = factors[0].shape[1]
        if outs is None:
            outs = [torch.empty((d, R), dtype=torch.float32, device=factors[0].device) for d in self.dims]
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        op = (c_voidp * self.nd)(*[_ptr(o) for o in outs])
        pl = Plan()
        check(lib().mmcsf_tune(self._h, R, self._dtype(factors), fp, op, _stream(stream), ctypes.byref(pl)))
        return self._plan_dict(pl)

    def tune_precision(self, factors, outs=None, error_budget=0.0, stream=None):
        """Per-mode precision plan for FP32 factors (mmcsf_tune_precision):
        every launch of mttkrp_all runs BF16 factor copies where that is faster
        and the mode's output moves by at most error_budget (relative
        Frobenius) against the FP32-factor output. Returns the plan with, per
        mode, "dtype", "bf16_error", "ms_f32", "ms_bf16"."""
        import torch
        R = factors[0].shape[1]
        if outs is None:
            outs = [torch.empty((d, R), dtype=torch.float32, device=factors[0].device) for d in self.dims]
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        op = (c_voidp * self.nd)(*[_ptr(o) for o in outs])
        pl = Plan()
        check(lib().mmcsf_tune_precision(self._h, R, fp, op, ctypes.c_double(error_budget), _stream(stream),
                                         ctypes.byref(pl)))
        return self._plan_dict(pl)

    def set_plan(self, plan):
        """Install a plan as returned by tune() / tune_precision() (JSON round
        trips allowed: string mode keys are accepted)."""
        pl = Plan()
        dt = {"f32": DTYPE_F32, "bf16": DTYPE_BF16}
        pl.factor_dtype = dt[plan.get("dtype", "f32")]
        pl.mixed = 1 if plan.get("mixed") else 0
        for m, e in plan.items():
            if m in ("dtype", "mixed", "fiber_threshold", "convert_ms"):
                continue
            if m == "pair":
                pl.pair = 1 if e.get("use") else 0
                pl.pair_chunk = e.get("chunk", 0)
                pl.pair_min_blocks = e.get("min_blocks", 0)
                pl.pair_kernel = e.get("kernel", 0)
                pl.pair_dtype = dt[e.get("dtype", "f32")]
                continue
            m = int(m)
            pl.traversal[m] = e["traversal"]
            pl.chunk[m] = e["chunk"]
            pl.min_blocks[m] = e.get("min_blocks", 0)
            pl.kernel[m] = e.get("kernel", 0)
            pl.mode_dtype[m] = dt[e.get("dtype", "f32")]
        check(lib().mmcsf_set_plan(self._h, ctypes.byref(pl)))

    def cpd(self, rank, max_iters=10, tol=1e-5, precision="fp32", init=None, seed=0, graph=True, stream=None,
            profile=False):
        """CP-ALS on the device (mmcsf_cpd). precision: "fp32" (FP32 factors and
        small-matrix math), "bf16" (BF16 factors, FP64 solve/fit) or
        "fp64solve" (FP32 factors, FP64 solve/fit). graph: the whole loop as one
        CUDA graph launch (on a side stream unless `stream` is given; the FP32
        forms run host-driven on the default stream); False: host-driven.
        init: optional list of FP32 CUDA tensors (dims[m] x rank). profile:
        time every phase (host-driven loop). Returns a dict with fit, iters,
        converged, seconds, history, lambda, factors (and phase_ms)."""
        import torch
        prec = {"fp32": 0, "bf16": 1, "fp64solve": 2}[precision]
        o = CpdOpts()
        o.rank = int(rank)
        o.max_iters = int(max_iters)
        o.tol = float(tol)
        o.precision = prec
        o.no_graph = 0 if graph else 1
        o.seed = int(seed)
        o.profile = 1 if profile else 0
        dev = init[0].device if init is not None else torch.device("cuda")
        outs = [torch.empty((d, rank), dtype=torch.float32, device=dev) for d in self.dims]
        ip = None
        if init is not None:
            keep = [t.contiguous().float() for t in init]
            ip = (c_voidp * self.nd)(*[_ptr(t) for t in keep])
        op = (c_voidp * self.nd)(*[_ptr(t) for t in outs])
        lam = (ctypes.c_double * rank)()
        res = CpdResult()
        st = stream
        if st is None:
            st = torch.cuda.Stream(device=dev) if graph else torch.cuda.current_stream(dev)
        cur = torch.cuda.current_stream(dev)
        if st != cur:
            st.wait_stream(cur)  # the initial factors (and their FP32 copies) come from the current stream
        check(lib().mmcsf_cpd(self._h, ctypes.byref(o), ip, op, lam, ctypes.byref(res), _stream(st)))
        torch.cuda.synchronize(dev)
        return {"fit": res.fit, "iters": res.iters, "converged": bool(res.converged), "seconds": res.seconds,
                "graph": bool(res.graph), "launches": res.launches,
                "history": [res.fit_history[i] for i in range(min(res.iters, len(res.fit_history)))],
                "lambda": np.array([lam[i] for i in range(rank)]), "factors": outs,
                "phase_ms": ({n: res.phase_ms[i] for i, n in enumerate(_lib.CPD_PHASE_NAMES)} if profile else None)}

    # -- sampled model and adjoint ------------------------------------------
    def partitioning(self):
        """(partition_rule, rounds the partition heuristic took to settle)."""
        rule, rounds = ctypes.c_int(), ctypes.c_int()
        check(lib().mmcsf_format_partitioning(self._h, ctypes.byref(rule), ctypes.byref(rounds)))
        return rule.value, rounds.value

    def partitions(self):
        """Indices of the non-empty parts (MM-CSF: partitions 0..nd-1), in
        the format's nonzero order."""
        if self.impl != IMPL_MMCSF:
            return [0]
        return [p for p in range(self.nd) if self.info(p)["present"]]

    def _main_part(self):
        if self.impl == IMPL_MMCSF:
            for p in range(self.nd):
                if self.info(p)["present"]:
                    return p
            return 0
        return 0

    def values(self):
        """Borrowed torch view of the tensor's values in the format's nonzero
        order (the order of sampled_model's output and cp_adjoint's grad)."""
        import torch
        vp = c_voidp()
        n = c_u64()
        check(lib().mmcsf_format_values(self._h, ctypes.byref(vp), ctypes.byref(n)))
        return torch.as_tensor(_CudaArray(vp.value, n.value, "<f4"), device="cuda")

    def nonzero_coords(self):
        """Per-mode coordinates (numpy uint64) of every nonzero in the
        format's nonzero order; needs keep_coo=True at build time."""
        parts = self.partitions() or [self._main_part()]
        return [np.concatenate([self.export(p, f"inds{m}") for p in parts]) for m in range(self.nd)]

    def sampled_model(self, factors, lam=None, out=None, stream=None):
        """xhat[x] = sum_r lam_r prod_m A_m[i_m(x), r] at every nonzero, in the
        format's nonzero order (float32 CUDA tensor of nnz entries)."""
        import torch
        R = factors[0].shape[1]
        if out is None:
            out = torch.empty(self.nnz, dtype=torch.float32, device=factors[0].device)
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        check(lib().mmcsf_sampled_model(self._h, R, self._dtype(factors), fp,
                                        _ptr(lam) if lam is not None else None, _ptr(out), _stream(stream)))
        return out

    def cp_adjoint(self, mode, factors, grad, lam=None, out=None, cfg=None, stream=None):
        """lam (.) MTTKRP of the tensor with this sparsity and values `grad`
        (nnz float32 in the format's nonzero order): the gradient of
        sum_x grad[x] * xhat[x] with respect to factor `mode`."""
        import torch
        R = factors[0].shape[1]
        if out is None:
            out = torch.empty((self.dims[mode], R), dtype=torch.float32, device=factors[0].device)
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        check(lib().mmcsf_cp_adjoint(self._h, mode, R, self._dtype(factors), fp,
                                     _ptr(lam) if lam is not None else None, _ptr(grad), _ptr(out),
                                     self._cfg(cfg), _stream(stream)))
        return out

    def poisson_step(self, factors, eps=1e-10, stream=None):
        """Fused Poisson step (mmcsf_poisson_step): returns (w, grad_root,
        loss, root_mode) with w[x] = y[x] / (xhat[x] + eps), loss =
        sum_x y[x] log(xhat[x] + eps) (a 1-element float64 CUDA tensor) and
        grad_root its gradient for the slice mode's factor."""
        import torch
        R = factors[0].shape[1]
        dev = factors[0].device
        root = ctypes.c_int()
        w = torch.empty(self.nnz, dtype=torch.float32, device=dev)
        order0 = self.info(self._main_part())["mode_order"][0]
        g = torch.empty((self.dims[order0], R), dtype=torch.float32, device=dev)
        loss = torch.empty(1, dtype=torch.float64, device=dev)
        fp = (c_voidp * self.nd)(*[_ptr(f) for f in factors])
        check(lib().mmcsf_poisson_step(self._h, R, self._dtype(factors), fp, ctypes.c_float(eps), _ptr(w), _ptr(g),
                                       _ptr(loss), ctypes.byref(root), _stream(stream)))
        return w, g, loss, root.value

    def ttm(self, factor, out=None, stream=None):
        """TTM along the leaf mode of a 3-D B-CSF format (mmcsf_ttm): one
        R-vector per leaf fiber, in the format's fiber order. factor: the
        leaf mode's factor (dims[leaf] x R, float32 or bfloat16, CUDA)."""
        import torch
        R = factor.shape[1]
        n = c_u64()
        check(lib().mmcsf_ttm(self._h, R, self._dtype([factor]), None, None, ctypes.byref(n), _stream(stream)))
        if out is None:
            out = torch.empty((int(n.value), R), dtype=torch.float32, device=factor.device)
        check(lib().mmcsf_ttm(self._h, R, self._dtype([factor]), _ptr(factor), _ptr(out), ctypes.byref(n),
                              _stream(stream)))
        return out

    @property
    def last_launches(self):
        n = ctypes.c_int()
        check(lib().mmcsf_format_last_launches(self._h, ctypes.byref(n)))
        return n.value


def autotune(coo, factors, impl=IMPL_MMCSF, mode=0, views=0, partition_rule=0, f_candidates=(0, 128, 32),
             error_budget=0.0, outs=None, stream=None, view_order=0):
    """Build the format for every fiber-split threshold in f_candidates (0 =
    no split), tune each (per-mode precision within error_budget for MM-CSF),
    and return (the fastest format, its plan) (mmcsf_autotune). factors: FP32
    CUDA tensors."""
    import torch
    nd, dims, _ = coo.info()
    R = factors[0].shape[1]
    if outs is None:
        outs = [torch.empty((d, R), dtype=torch.float32, device=factors[0].device) for d in dims]
    o = BuildOpts()
    o.impl, o.mode, o.views, o.partition_rule = impl, mode, int(views), int(partition_rule)
    o.view_order = int(view_order)
    fc = (c_u64 * len(f_candidates))(*[int(f) for f in f_candidates])
    fp = (c_voidp * nd)(*[_ptr(f) for f in factors])
    op = (c_voidp * nd)(*[_ptr(x) for x in outs])
    h = c_voidp()
    pl = Plan()
    check(lib().mmcsf_autotune(coo._h, ctypes.byref(o), fc, len(f_candidates), R, fp, op, ctypes.c_double(error_budget),
                               _stream(stream), ctypes.byref(h), ctypes.byref(pl)))
    F = Format.__new__(Format)
    F._h = h
    F.impl = impl
    F.mode = mode
    F.nd, F.dims, F.nnz = coo.info()
    return F, F._plan_dict(pl)


class _CudaArray:
    """Minimal __cuda_array_interface__ wrapper around a raw device pointer."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr or 0), False),
                                         "version": 2}


def _host_ptr(a):
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"] or a.dtype != np.float32:
            raise MmcsfError(1, "host factors must be C-contiguous float32")
        return a.ctypes.data
    return a.data_ptr()  # torch CPU tensor (possibly pinned)
