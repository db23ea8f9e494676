"""ctypes binding to the in-tree C ABI (include/mmcsf.h, lib/libmmcsf.so).

Loading fails loudly: there is no CPU fallback for anything in this package.
"""
import ctypes
import os

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# MMCSF_LIBRARY selects another in-tree build, e.g. lib/libmmcsf_bounds.so
# (every compute entry point validates a format once before launching on it)
LIB_PATH = os.environ.get("MMCSF_LIBRARY") or os.path.join(_PKG_ROOT, "lib", "libmmcsf.so")

c_u64 = ctypes.c_uint64
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_voidp = ctypes.c_void_p
c_int = ctypes.c_int


class MmcsfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class GenSpec(ctypes.Structure):
    _fields_ = [("nd", c_int), ("dims", c_u64 * 4), ("nnz", c_u64), ("dist", c_int * 4),
                ("zipf_s", ctypes.c_double * 4), ("val_dist", c_int), ("seed", c_u64), ("planted_rank", c_int),
                ("noise", ctypes.c_double), ("poisson", c_int)]


class BuildOpts(ctypes.Structure):
    _fields_ = [("impl", c_int), ("mode", c_int), ("fiber_threshold", c_u64), ("partition_rule", c_int),
                ("keep_coo", c_int), ("views", c_int), ("partition_ratio", c_int), ("view_order", c_int)]


class PartInfo(ctypes.Structure):
    _fields_ = [("present", c_int), ("nd", c_int), ("mode_order", c_int * 4), ("nnz", c_u64),
                ("n_slices", c_u64), ("n_fbrs", c_u64), ("n_fibers", c_u64), ("device_bytes", c_u64)]


class KernelCfg(ctypes.Structure):
    _fields_ = [("chunk", c_int), ("block_threads", c_int), ("traversal", c_int), ("min_blocks", c_int),
                ("kernel", c_int), ("reserved", c_int * 3)]


class Plan(ctypes.Structure):
    _fields_ = [("traversal", c_int * 4), ("chunk", c_int * 4), ("min_blocks", c_int * 4),
                ("kernel", c_int * 4), ("ms", ctypes.c_float * 4), ("pair", c_int), ("pair_chunk", c_int),
                ("pair_min_blocks", c_int), ("pair_kernel", c_int),
                ("pair_ms", ctypes.c_float), ("factor_dtype", c_int), ("mixed", c_int), ("mode_dtype", c_int * 4),
                ("pair_dtype", c_int), ("bf16_error", ctypes.c_float * 4), ("ms_f32", ctypes.c_float * 4),
                ("ms_bf16", ctypes.c_float * 4), ("pair_ms_f32", ctypes.c_float), ("pair_ms_bf16", ctypes.c_float),
                ("convert_ms", ctypes.c_float), ("fiber_threshold", c_int)]


class CpdOpts(ctypes.Structure):
    _fields_ = [("rank", c_int), ("max_iters", c_int), ("tol", ctypes.c_double), ("precision", c_int),
                ("no_graph", c_int), ("seed", c_u64), ("profile", c_int)]


CPD_MAX_HISTORY = 1000
CPD_PHASES = 6
CPD_PHASE_NAMES = ("mttkrp", "solve", "apply", "lambda", "finish", "fit")


class CpdResult(ctypes.Structure):
    _fields_ = [("iters", c_int), ("converged", c_int), ("graph", c_int), ("launches", c_int),
                ("fit", ctypes.c_double), ("seconds", ctypes.c_double),
                ("phase_ms", ctypes.c_double * CPD_PHASES),
                ("fit_history", ctypes.c_double * CPD_MAX_HISTORY)]


_lib = None

# (name, argtypes) for every exported entry point in include/mmcsf.h
SIGNATURES = {
    "mmcsf_status_string": ([c_int], ctypes.c_char_p),
    "mmcsf_last_error": ([], ctypes.c_char_p),
    "mmcsf_version": ([], c_int),
    "mmcsf_coo_load_tns": ([ctypes.c_char_p, ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_coo_create": ([c_int, c_u64p, c_u64, ctypes.POINTER(c_u32p), c_f32p, ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_coo_create_device": ([c_int, c_u64p, c_u64, ctypes.POINTER(c_voidp), c_voidp, c_voidp,
                                 ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_coo_info": ([c_voidp, ctypes.POINTER(c_int), c_u64p, c_u64p], c_int),
    "mmcsf_coo_to_host": ([c_voidp], c_int),
    "mmcsf_coo_to_device": ([c_voidp, c_voidp], c_int),
    "mmcsf_coo_host_arrays": ([c_voidp, ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_coo_device_arrays": ([c_voidp, ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_coo_write_tns": ([c_voidp, ctypes.c_char_p], c_int),
    "mmcsf_coo_destroy": ([c_voidp], None),
    "mmcsf_generate": ([ctypes.POINTER(GenSpec), c_voidp, ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_build": ([c_voidp, ctypes.POINTER(BuildOpts), c_voidp, ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_format_destroy": ([c_voidp], None),
    "mmcsf_format_info": ([c_voidp, c_int, ctypes.POINTER(PartInfo)], c_int),
    "mmcsf_format_meta": ([c_voidp, ctypes.POINTER(c_int), ctypes.POINTER(c_int)], c_int),
    "mmcsf_format_partitioning": ([c_voidp, ctypes.POINTER(c_int), ctypes.POINTER(c_int)], c_int),
    "mmcsf_format_export": ([c_voidp, c_int, ctypes.c_char_p, c_u64p, c_u64, c_u64p], c_int),
    "mmcsf_format_export_f32": ([c_voidp, c_int, ctypes.c_char_p, c_f32p, c_u64, c_u64p], c_int),
    "mmcsf_mttkrp": ([c_voidp, c_int, c_int, c_int, ctypes.POINTER(c_voidp), c_voidp,
                      ctypes.POINTER(KernelCfg), c_voidp], c_int),
    "mmcsf_mttkrp_all": ([c_voidp, c_int, c_int, ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp),
                          ctypes.POINTER(KernelCfg), c_voidp], c_int),
    "mmcsf_mttkrp_all_host": ([c_voidp, c_int, ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp),
                               ctypes.POINTER(KernelCfg), c_voidp], c_int),
    "mmcsf_format_last_launches": ([c_voidp, ctypes.POINTER(c_int)], c_int),
    "mmcsf_format_check": ([c_voidp, c_u64p, c_voidp], c_int),
    "mmcsf_tune": ([c_voidp, c_int, c_int, ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp), c_voidp,
                    ctypes.POINTER(Plan)], c_int),
    "mmcsf_set_plan": ([c_voidp, ctypes.POINTER(Plan)], c_int),
    "mmcsf_tune_precision": ([c_voidp, c_int, ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp), ctypes.c_double,
                              c_voidp, ctypes.POINTER(Plan)], c_int),
    "mmcsf_autotune": ([c_voidp, ctypes.POINTER(BuildOpts), c_u64p, c_int, c_int, ctypes.POINTER(c_voidp),
                        ctypes.POINTER(c_voidp), ctypes.c_double, c_voidp, ctypes.POINTER(c_voidp),
                        ctypes.POINTER(Plan)], c_int),
    "mmcsf_cpd": ([c_voidp, ctypes.POINTER(CpdOpts), ctypes.POINTER(c_voidp), ctypes.POINTER(c_voidp),
                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(CpdResult), c_voidp], c_int),
    "mmcsf_sampled_model": ([c_voidp, c_int, c_int, ctypes.POINTER(c_voidp), c_voidp, c_voidp, c_voidp], c_int),
    "mmcsf_cp_adjoint": ([c_voidp, c_int, c_int, c_int, ctypes.POINTER(c_voidp), c_voidp, c_voidp, c_voidp,
                          ctypes.POINTER(KernelCfg), c_voidp], c_int),
    "mmcsf_format_values": ([c_voidp, ctypes.POINTER(c_voidp), c_u64p], c_int),
    "mmcsf_probe_gather": ([c_voidp, c_u64, c_voidp, c_u64, c_int, c_int, ctypes.POINTER(ctypes.c_float), c_voidp],
                           c_int),
    "mmcsf_probe_gather_tma": ([c_voidp, c_u64, c_voidp, c_u64, c_int, c_int, c_int, c_int,
                                ctypes.POINTER(ctypes.c_float), c_voidp], c_int),
    "mmcsf_coo_write_bin": ([c_voidp, ctypes.c_char_p], c_int),
    "mmcsf_coo_load_bin": ([ctypes.c_char_p, ctypes.POINTER(c_voidp)], c_int),
    "mmcsf_poisson_step": ([c_voidp, c_int, c_int, ctypes.POINTER(c_voidp), ctypes.c_float, c_voidp, c_voidp,
                            c_voidp, ctypes.POINTER(c_int), c_voidp], c_int),
    "mmcsf_ttm": ([c_voidp, c_int, c_int, c_voidp, c_voidp, c_u64p, c_voidp], c_int),
    "mmcsf_mttkrp_pair": ([c_voidp, c_int, c_int, ctypes.POINTER(c_voidp), c_voidp, c_voidp, ctypes.POINTER(c_int),
                           ctypes.POINTER(KernelCfg), c_voidp], c_int),
    "mmcsf_mttkrp_coo_host": ([c_voidp, c_int, c_int, ctypes.POINTER(c_voidp), c_voidp, c_int], c_int),
    "mmcsf_sort_coo_noalloc": ([c_int, c_int, c_int, c_u64p, c_u64, ctypes.POINTER(c_voidp), c_voidp,
                                ctypes.POINTER(c_voidp), c_voidp, c_voidp], c_int),
}


def lib():
    """The loaded library. Raises if the in-tree build is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MmcsfError(-1, f"{LIB_PATH} is missing: build it with `make -C mm-csf_b200` "
                                 "(python -c 'import __graft_entry__ as g; g.build()')")
        L = ctypes.CDLL(LIB_PATH)
        for name, (argt, rest) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = argt
            fn.restype = rest
        _lib = L
    return _lib


def check(status):
    if status != 0:
        L = lib()
        raise MmcsfError(status, L.mmcsf_last_error().decode() or L.mmcsf_status_string(status).decode())
    return status
