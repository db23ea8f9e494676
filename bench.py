#!/usr/bin/env python3
"""All-mode MTTKRP benchmark (MM-CSF, B200).

Workload (default): 3-mode tensor 500,000 x 2,000,000 x 20,000 with 100M
nonzeros, every mode index Zipf(s=1.1) after a seeded permutation, values
lognormal(0,1), rank R=32 FP32 factors uniform in [0,1); MM-CSF format
(-t 12, -m 0, no fiber split). A step is one all-mode MTTKRP (every mode from
the same input factors), the reference's MTTKRP_MIHCSR_GPU loop.

value      = effective HBM GB/s over all ranks: the MM-CSF traversal's
             algorithmic bytes per all-mode MTTKRP (structure read once per
             mode, every touched factor row once, the dense output written
             once) / device time per step.
e2e        = the same bytes / time of the host-buffer C-ABI call
             (mmcsf_mttkrp_all_host: factors H2D, all modes, outputs D2H).
units      = the step's launches as mmcsf_mttkrp_all issues them under the
             tuned plan (the two-output walk for the partition's slice and
             middle modes when it wins, one MTTKRP per other mode), each with
             its CUDA-event time and algorithmic bytes.
roofline   = the dominant launch's kernel: its algorithmic bytes / its average
             CUDA-event duration, against MEASURED_PEAKS.json's HBM copy rate;
             its DRAM traffic from the committed ncu summary; the row-gather
             ceiling measured on the same GPU (mmcsf_probe_gather).
cpu_baseline / --impl reference = the reference's own MTTKRP_COO_CPU
             (oracle/_ref) over every nonzero on all host threads (contiguous
             nonzero ranges, private outputs added in the step), each step
             timed whole, no sample; the reference arm builds its tensor with
             the host restatement of the generator (oracle/generate.c) and
             loads nothing of the CUDA library.
error_vs_fp64 = every output of the timed step against an FP64 MTTKRP of
             the same factors (largest |d| / (|ref| + 1e-6 max|ref|), and the
             relative Frobenius norm).
reference_gpu = the reference's own GPU MTTKRP (MTTKRP_MIHCSR_GPU, built for
             sm_100a) on this GPU and the same arrays, at its defaults and
             its benchmark script's settings, beside this step.
also       = format_build_ms (device construction), bf16_factors (the step
             with BF16 factors, tuned, and its errors), r64 (the same
             workload at R = 64, FP32 and BF16), autotune (the tuner choosing
             -f and each mode's factor precision), config1 (1000^3 uniform,
             -f 128 -w 1: device, the library's host -t 1 path and the
             reference's CPU path), skewed4d (the 4-D workload: MM-CSF all
             modes against B-CSF and HB-CSF per mode), ttm (the reference's
             ttm on the same tensor), cp (CP-ALS and Poisson gradient CP:
             BF16 vs FP32 seconds per iteration and fits),
             partition_heuristic (the same step on the partitions the
             reference's heuristic picks, partition_rule 1).

--gpus N > 1 (torchrun) = ONE tensor row-sharded across the ranks: every
             mode's rows are split by nonzero count, each rank runs the
             MTTKRP of its rows of every mode on single-mode CSFs of its
             shards, no collective in the step (mmcsf.dist; strong scaling,
             max over ranks). --sharded runs that path on one GPU too.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "mm-csf_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "all-mode MTTKRP ms & HBM GB/s (effective GB/s = MM-CSF algorithmic bytes / all-mode time)"

WORKLOADS = {
    "skewed3d": dict(dims=[500000, 2000000, 20000], nnz=100_000_000, dist=[1, 1, 1], zipf=1.1, val=1, R=32,
                     desc="500000x2000000x20000, 100M nnz, Zipf(1.1) per mode, lognormal values, R=32"),
    "uniform3d": dict(dims=[1000, 1000, 1000], nnz=100_000, dist=[0, 0, 0], zipf=1.0, val=0, R=32,
                      desc="1000^3, 100k uniform nnz, R=32"),
    "cpals3d": dict(dims=[200000, 200000, 200000], nnz=50_000_000, dist=[0, 0, 0], zipf=1.0, val=0, R=16, views=2,
                    desc="200000^3, 50M uniform nnz, R=16: the CP-ALS tensor's index structure (values uniform), "
                         "every mode through its view"),
    "skewed4d": dict(dims=[1000000, 20000, 5000, 200], nnz=140_000_000, dist=[1, 1, 1, 0], zipf=1.0, val=2, R=32,
                     views=2,
                     desc="1000000x20000x5000x200, 140M nnz, Zipf(1.0) modes 0-2, uniform mode 3, integer values "
                          "1-50, R=32; B-CSF / HB-CSF per mode beside MM-CSF all modes"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="skewed3d", choices=list(WORKLOADS))
    ap.add_argument("--nnz", type=int, default=0, help="override nonzero count (profiling on a small case)")
    ap.add_argument("--rank", type=int, default=0, help="override R")
    ap.add_argument("--fiber-threshold", type=int, default=0)
    ap.add_argument("--dtype", default="f32", choices=["f32", "bf16"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--views", type=int, default=None,
                    help="0 none, 1 leaf-level modes, 2 every mode (default: the workload's)")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--plan-file", default="",
                    help="JSON plan (as printed by a tuned run) to use instead of tuning: a file, or the JSON itself")
    ap.add_argument("--no-cp", action="store_true", help="skip the CP-ALS and Poisson gradient-CP sections")
    ap.add_argument("--no-formats", action="store_true", help="4-D workloads: skip the B-CSF / HB-CSF section")
    ap.add_argument("--no-bf16", action="store_true", help="skip the BF16-factor section")
    ap.add_argument("--no-heuristic", action="store_true",
                    help="skip the section on the partition heuristic's MM-CSF (partition_rule 1)")
    ap.add_argument("--cp-scale", type=float, default=1.0, help="scale the CP workloads' nonzero counts")
    ap.add_argument("--no-r64", action="store_true", help="skip the R=64 section of the skewed 3-D workload")
    ap.add_argument("--no-config1", action="store_true", help="skip the 1000^3 uniform (config 1) section")
    ap.add_argument("--no-4d", action="store_true", help="skip the 4-D (B-CSF / HB-CSF / MM-CSF) section")
    ap.add_argument("--no-autotune", action="store_true", help="skip the -f / precision autotuner section")
    ap.add_argument("--no-refgpu", action="store_true", help="skip the reference's own GPU MTTKRP on this GPU")
    ap.add_argument("--sharded", action="store_true",
                    help="run the row-sharded multi-GPU path (the default for --gpus N > 1) also on one GPU")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(workload, R, dtype, mode, kernel):
    """DRAM bytes per launch of one mode's MTTKRP kernel from a committed ncu
    summary (lines `mode<m>: <kernel> <bytes>`), or None when the summary has
    no entry for that mode and kernel."""
    p = os.path.join(ROOT, "profiles", f"traffic_{workload}_R{R}_{dtype}.txt")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        for line in fh:
            f = line.split()
            if len(f) == 3 and f[0] == f"mode{mode}:" and f[1] == kernel:
                return float(f[2])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r for r in csv.reader(io.StringIO(out)) if len(r) >= 9]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for i, n in enumerate(names):
                if r[5 + i].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def struct_bytes(nd, nnz, nfib, nfbrs):
    """Structure bytes one traversal of a CSF part reads: vals + leaf index per
    nonzero; per leaf fiber its pointer, index and slice map (3-D), plus the
    fiber->fbrS map per fiber and fbrS index + slice map per fbrS (4-D)."""
    return nnz * 8 + (nfib * 12 if nd == 3 else nfib * 12 + nfbrs * 8)


def mode_bytes(nd, dims, m, R, esz, sbytes, rows_touched):
    """Compulsory bytes of one mode's MTTKRP: the traversal's structure, every
    touched row of the other factors once, the dense output written once."""
    fact = sum(rows_touched[q] * R * esz for q in range(nd) if q != m)
    return sbytes + fact + dims[m] * R * 4


def workload_stats(inds_dev, dims, order):
    """Rows touched per mode and fiber count (no split) with torch ops."""
    import torch
    rows = [int(torch.unique(i).numel()) for i in inds_dev]
    key = inds_dev[order[0]].long()
    for q in order[1:len(order) - 1]:  # leaf fibers: distinct prefixes of all but the leaf level
        key = key * dims[q] + inds_dev[q].long()
    nfib = int(torch.unique(key).numel())
    return rows, nfib


def device_coo(X):
    """Device index arrays of a CooTensor as torch int32 tensors (copies)."""
    inds, vals = X.device_tensors()
    return [i.clone() for i in inds], vals.clone()


def host_threads():
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class RefCpuMttkrp:
    """All-mode MTTKRP with the reference's own MTTKRP_COO_CPU
    (src/mttkrp_cpu.cpp:60-113, built as oracle/_ref; the C restatement of the
    oracle when the reference was not built here) over ALL nonzeros on
    `threads` host threads: thread t runs it on the t-th contiguous range of
    the nonzeros into a private zeroed output, and the step also adds the
    private outputs (rows split across the threads). The function is serial
    as shipped (its OpenMP pragma is commented out, src/mttkrp_cpu.cpp:79), so
    the threads split the nonzeros among calls."""

    def __init__(self, inds_host, vals_host, dims, R, threads):
        import ctypes
        import numpy as np

        from oracle import oracle as O
        self.kind = "reference" if O.ref_available() else "port"
        self.lib = O.ref_lib() if self.kind == "reference" else O.lib()
        self.dims, self.R, self.nd = list(dims), R, len(dims)
        n = len(vals_host)
        self.n = n
        # bound the private outputs at about 24 GB
        per = max(dims) * R * 4
        self.T = max(1, min(threads, n, (24 << 30) // max(1, per)))
        rng = np.random.default_rng(0)
        self.U = [rng.random((d, R)).astype(np.float32) for d in dims]
        cuts = [n * t // self.T for t in range(self.T + 1)]
        self.parts = []
        fp = ctypes.POINTER(ctypes.c_float)
        for t in range(self.T):
            a, b = cuts[t], cuts[t + 1]
            ind = [np.ascontiguousarray(i[a:b], dtype=np.uint64) for i in inds_host]
            v = np.ascontiguousarray(vals_host[a:b])
            outs = [np.zeros((d, R), np.float32) for d in dims]
            self.parts.append((ind, v, outs, O._ptr_array(ind), v.ctypes.data_as(fp)))
        self.out = [np.zeros((d, R), np.float32) for d in dims]
        self.dptr = (ctypes.c_uint64 * self.nd)(*[int(d) for d in dims])
        self.fp = fp

    def _run(self, t, m):
        import ctypes
        ind, v, outs, ip, vp = self.parts[t]
        outs[m].fill(0.0)
        fac = (self.fp * self.nd)(*[(outs[m] if q == m else self.U[q]).ctypes.data_as(self.fp)
                                    for q in range(self.nd)])
        if self.kind == "reference":
            rc = self.lib.ref_coo_mttkrp(self.nd, self.dptr, ctypes.c_uint64(len(v)), ip, vp, m, self.R, fac)
            assert rc == 0
        else:
            self.lib.orc_mttkrp_coo_f32(self.nd, ctypes.c_uint64(len(v)), ip, vp, m, self.R, fac)

    def _sum(self, t, m):
        rows = self.dims[m]
        a, b = rows * t // self.T, rows * (t + 1) // self.T
        acc = self.out[m][a:b]
        acc[:] = self.parts[0][2][m][a:b]
        for u in range(1, self.T):
            acc += self.parts[u][2][m][a:b]

    def step(self):
        """One all-mode MTTKRP over every nonzero (threads, then the sums)."""
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(self.T) as ex:
            for m in range(self.nd):
                list(ex.map(lambda t: self._run(t, m), range(self.T)))
                list(ex.map(lambda t: self._sum(t, m), range(self.T)))

    def seconds(self):
        t = time.perf_counter()
        self.step()
        return time.perf_counter() - t


CPALS = dict(dims=[200000, 200000, 200000], nnz=50_000_000, planted=16, noise=0.01, R=16, max_iters=50, tol=1e-5,
             desc="200000^3, 50M uniform nnz, planted rank-16 CP (factors U[0,1)) + Gaussian noise 0.01 RMS, R=16, "
                  "tol 1e-5 on fit change, at most 50 iterations")
GCP = dict(dims=[100000, 50000, 10000], nnz=20_000_000, zipf=1.05, planted=32, R=32, iters=150, lr=0.05,
           desc="100000x50000x10000, 20M nnz, Zipf(1.05) per mode, Poisson counts of a planted nonnegative "
                "rank-32 CP, R=32, projected Adam (step 0.05 x mean initial entry, initial mass = data mass) on the Poisson "
                "loss over every entry")


def format_section(X, dims, R, U, rows, hbm_peak, refs=None):
    """Single-mode B-CSF (-t 8) and HB-CSF (-t 10) MTTKRP for every mode, each
    format built for that mode and tuned, timed like the MM-CSF steps: per
    mode its time, algorithmic bytes (the traversal's structure, the touched
    rows of the other factors, the output once), the fraction of the HBM
    roofline, and (with `refs`, FP64 outputs per mode) the error against the
    FP64 oracle."""
    import torch
    import mmcsf
    out = {}
    nd = len(dims)
    esz = U[0].element_size()
    for name, impl in (("bcsf", mmcsf.IMPL_BCSF), ("hbcsf", mmcsf.IMPL_HBCSF)):
        ms, gbs, errs = [], [], []
        for m in range(nd):
            F = mmcsf.Format(X, impl=impl, mode=m)
            o = torch.empty(dims[m], R, device="cuda")
            outs = [o if q == m else torch.empty(1, R, device="cuda") for q in range(nd)]
            plan = F.tune(U, outs)
            for _ in range(3):
                F.mttkrp(m, U, o)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                F.mttkrp(m, U, o)
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 10
            ms.append(t)
            pi = F.info(0)
            kern = plan[m].get("kernel") if plan else None
            if kern == 3 and pi["mode_order"].index(m) in (0, nd - 1):
                sb = X.nnz * (12 if nd == 3 else 16) + pi["n_slices"] * 8
            else:
                sb = struct_bytes(nd, X.nnz, pi["n_fibers"], pi["n_fbrs"])
            b = mode_bytes(nd, dims, m, R, esz, sb, rows)
            gbs.append(b / (t / 1e3) / 1e9)
            if refs:
                errs.append(err_vs(o, refs[m]))
            del F
            torch.cuda.empty_cache()
        out[name] = {"mode_ms": ms, "all_mode_ms": sum(ms), "mode_gbs": gbs,
                     "mode_roofline_frac": [g / hbm_peak for g in gbs], "error_vs_fp64": errs or None}
    return out


def heuristic_section(X, dims, R, tdt, views):
    """The same all-mode step on the MM-CSF whose partitions the reference's
    partition heuristic chooses (partition_rule 1, -h 1) instead of the
    shipped all-to-partition-2: device build time (the heuristic's rounds
    included), partition sizes, and the tuned step time."""
    import torch
    import mmcsf
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, views=views, partition_rule=1)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    _, rounds = F.partitioning()
    parts = {p: F.info(p)["nnz"] for p in F.partitions()}
    g = torch.Generator(device="cuda").manual_seed(1234)
    U = [torch.rand(d, R, device="cuda", generator=g).to(tdt) for d in dims]
    outs = [torch.empty(d, R, device="cuda") for d in dims]
    F.tune(U, outs)
    for _ in range(3):
        F.mttkrp_all(U, outs)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(10):
        F.mttkrp_all(U, outs)
    e1.record()
    torch.cuda.synchronize()
    out = {"format_build_ms": build_ms, "rounds": rounds, "partition_nnz": parts,
           "ms_per_step": e0.elapsed_time(e1) / 10, "launches_per_step": F.last_launches}
    del F
    torch.cuda.empty_cache()
    return out


def step_units(F, U, outs, plan):
    """The launches of one all-mode step as mmcsf_mttkrp_all issues them under
    `plan`: the two-output walk for the partition's slice and middle modes
    when the plan chose it, one MTTKRP per remaining mode. Returns
    [(modes, fn)]; timing each fn separately gives the per-kernel times."""
    nd = len(U)
    units = []
    done = set()
    if plan and plan.get("pair", {}).get("use"):
        m0, m1 = F.pair_modes()
        po = {m0: outs[m0], m1: outs[m1]}
        units.append(((m0, m1), lambda: F.mttkrp_pair(U, po)))
        done = {m0, m1}
    for m in range(nd):
        if m not in done:
            units.append(((m,), lambda m=m: F.mttkrp(m, U, outs[m])))
    return units


def time_units(units, steps, stream=None):
    """Per-unit device times (CUDA events on the launching stream), mean over
    `steps` steps, and the whole span."""
    import torch
    stream = stream or torch.cuda.current_stream()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(units) + 1)] for _ in range(steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for k in range(steps):
        ev[k][0].record(stream)
        for i, (_, fn) in enumerate(units):
            fn()
            ev[k][i + 1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    unit_ms = [statistics.mean(ev[k][i].elapsed_time(ev[k][i + 1]) for k in range(steps)) for i in range(len(units))]
    return unit_ms, t0.elapsed_time(t1)


def fp64_mttkrp(inds_dev, vals_dev, U, mode, chunk=1 << 23):
    """FP64 MTTKRP of one mode from the COO nonzeros (torch on the device,
    outside every timed region): the precision oracle the benchmarked outputs
    are compared with. U: the factors as the kernels read them (FP32 or BF16)."""
    import torch
    nd = len(U)
    R = U[0].shape[1]
    out = torch.zeros(U[mode].shape[0], R, dtype=torch.float64, device="cuda")
    U64 = [u.double() if q != mode else None for q, u in enumerate(U)]
    n = vals_dev.numel()
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        p = vals_dev[a:b].double().unsqueeze(1).repeat(1, R)
        for q in range(nd):
            if q != mode:
                p *= U64[q].index_select(0, inds_dev[q][a:b].long())
        out.index_add_(0, inds_dev[mode][a:b].long(), p)
    del U64
    return out


def err_vs(out, ref):
    """Error of an output against its FP64 oracle: the largest elementwise
    |out - ref| / (|ref| + 1e-6 max|ref|) and the relative Frobenius norm."""
    d = out.double() - ref
    scale = float(ref.abs().max())
    return {"max_rel": float((d.abs() / (ref.abs() + 1e-6 * scale)).max()),
            "frobenius_rel": float(d.norm() / ref.norm())}


def bf16_section(F, U32, outs32, steps, warmup, inds_dev, vals_dev, refs32):
    """The same step with BF16 factors (FP32 accumulation), tuned for them:
    its time, its error against the FP64 MTTKRP of the same BF16 factors (the
    kernels' arithmetic), against the FP64 MTTKRP of the FP32 factors (that
    plus the factors' rounding), and against the FP32-factor outputs."""
    import torch
    U = [u.to(torch.bfloat16) for u in U32]
    outs = [torch.empty_like(o) for o in outs32]
    plan = F.tune(U, outs)
    for _ in range(warmup):
        F.mttkrp_all(U, outs)
    units = step_units(F, U, outs, plan)
    unit_ms, span = time_units(units, steps)
    F.mttkrp_all(U, outs)
    torch.cuda.synchronize()
    e_same, e_f32, e_out = [], [], []
    for m, (o, r) in enumerate(zip(outs, outs32)):
        ref_b = fp64_mttkrp(inds_dev, vals_dev, U, m)
        e_same.append(err_vs(o, ref_b))
        del ref_b
        e_f32.append(err_vs(o, refs32[m]))
        e_out.append(err_vs(o, r.double()))
    return {"ms_per_step": span / steps, "units": [{"modes": list(u[0]), "ms": t} for u, t in zip(units, unit_ms)],
            "plan": plan, "error_vs_fp64_same_factors": e_same, "error_vs_fp64_fp32_factors": e_f32,
            "error_vs_fp32_factor_outputs": e_out,
            "note": "BF16-rounded factor rows, FP32 products and accumulation; against the FP32 factors the "
                    "error is the factors' rounding"}


def ttm_section(X, dims, R, mode, rows_touched):
    """TTM along the leaf mode of the B-CSF format of `mode` (the reference's
    ttm): device time per call and its algorithmic GB/s (values + leaf index
    per nonzero, the touched leaf rows once, Y written once)."""
    import torch
    import mmcsf
    F = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=mode)
    leaf = F.info(0)["mode_order"][2]
    g = torch.Generator(device="cuda").manual_seed(5)
    U = torch.rand(dims[leaf], R, device="cuda", generator=g)
    Y = F.ttm(U)
    for _ in range(3):
        F.ttm(U, Y)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        F.ttm(U, Y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    nnz, nfib = F.nnz, Y.shape[0]
    b = nnz * 8 + rows_touched[leaf] * R * 4 + nfib * R * 4
    return {"mode": mode, "leaf_mode": leaf, "fibers": nfib, "ms": ms, "algorithmic_bytes": b,
            "gbs": b / (ms / 1e3) / 1e9}


def cp_section(seed, scale):
    """CP seconds per iteration to a fixed fit: BF16 factors (+ FP64 solve and
    fit) against plain FP32 CP-ALS, both with the whole loop in one CUDA graph
    (so the ratio isolates precision), the host-driven FP32 loop beside them,
    and Poisson gradient CP (sampled model + adjoint) with BF16 vs FP32
    factors."""
    import torch
    import mmcsf
    from mmcsf import gcp
    out = {}
    # ---- CP-ALS
    c = CPALS
    nnz = int(c["nnz"] * scale)
    X = mmcsf.CooTensor.generate(c["dims"], nnz, dist=[0, 0, 0], val_dist=mmcsf.VAL_UNIFORM01, seed=seed + 11,
                                 planted_rank=c["planted"], noise=c["noise"])
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=2)  # every mode can run as a slice level
    del X
    g = torch.Generator(device="cuda").manual_seed(seed + 5)
    R = c["R"]
    init = [torch.rand(d, R, device="cuda", generator=g) for d in c["dims"]]
    runs = {}
    for name in ("fp32", "fp32_host", "bf16", "fp64solve"):
        prec, graph = ("fp32", False) if name == "fp32_host" else (name, True)
        F.tune([t.to(torch.bfloat16) for t in init] if prec == "bf16" else init)  # plan for this factor type
        F.cpd(R, max_iters=2, tol=c["tol"], precision=prec, init=init, graph=graph)  # warm-up (tables, graph code)
        r = F.cpd(R, max_iters=c["max_iters"], tol=c["tol"], precision=prec, init=init, graph=graph)
        fx = F.cpd(R, max_iters=c["max_iters"], tol=1e-15, precision=prec, init=init, graph=graph)  # every iteration
        pr = F.cpd(R, max_iters=20, tol=1e-15, precision=prec, init=init, profile=True)  # per-phase times
        runs[name] = {"seconds_to_converge": r["seconds"], "iters_to_converge": r["iters"], "fit": r["fit"],
                      "converged": r["converged"], "graph": r["graph"], "launches": r["launches"],
                      "fixed_iters": fx["iters"], "fixed_seconds": fx["seconds"],
                      "s_per_iter": fx["seconds"] / max(1, fx["iters"]), "fixed_fit": fx["fit"],
                      "phase_ms_per_iter": {k: v / pr["iters"] for k, v in pr["phase_ms"].items()},
                      "phase_note": "host-driven profiled run (events at every phase boundary), 20 iterations"}
    f32, b16 = runs["fp32"], runs["bf16"]
    out["cp_als"] = {"workload": c["desc"] + (f" (nnz scaled to {nnz})" if scale != 1.0 else ""),
                     "runs": runs, "fit_gap_bf16_vs_fp32": abs(b16["fit"] - f32["fit"]),
                     "fit_gap_bf16_vs_fp64solve": abs(b16["fit"] - runs["fp64solve"]["fit"]),
                     "speedup_time_to_fit_bf16_vs_fp32": f32["seconds_to_converge"] / b16["seconds_to_converge"],
                     "speedup_s_per_iter_bf16_vs_fp32": f32["s_per_iter"] / b16["s_per_iter"],
                     "speedup_s_per_iter_bf16_vs_fp32_host": runs["fp32_host"]["s_per_iter"] / b16["s_per_iter"],
                     "note": "fp32 and bf16 both run the loop as one CUDA graph; fp32_host is the host-driven FP32 loop"}
    del F, init
    torch.cuda.empty_cache()
    # ---- Poisson gradient CP
    c = GCP
    nnz = int(c["nnz"] * scale)
    X = mmcsf.CooTensor.generate(c["dims"], nnz, dist=[1, 1, 1], zipf_s=c["zipf"], seed=seed + 13,
                                 planted_rank=c["planted"], poisson=True)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=2)
    del X
    R = c["R"]
    g = torch.Generator(device="cuda").manual_seed(seed + 7)
    init = [torch.rand(d, R, device="cuda", generator=g) * 0.5 + 0.25 for d in c["dims"]]
    runs = {}
    for prec in ("fp32", "bf16"):
        F.tune([t.to(torch.bfloat16) for t in init] if prec == "bf16" else init)  # plan for this factor type
        gcp.gcp_poisson(F, R, iters=3, lr=c["lr"], precision=prec, init=init)  # warm-up
        r = gcp.gcp_poisson(F, R, iters=c["iters"], lr=c["lr"], precision=prec, init=init)
        pr = gcp.gcp_poisson(F, R, iters=20, lr=c["lr"], precision=prec, init=init, profile=True)
        runs[prec] = {"ms_per_iter": r["ms"][-1] / r["iters"], "iters": r["iters"], "loss_first": r["loss"][0],
                      "loss_final": r["loss"][-1], "ms": r["ms"], "loss": r["loss"],
                      "phase_ms_per_iter": {k: v / pr["iters"] for k, v in pr["phase_ms"].items()}}
    f32, b16 = runs["fp32"], runs["bf16"]
    target = f32["loss_final"] * (1 + 1e-4)
    t_b16 = next((t for t, l in zip(b16["ms"], b16["loss"]) if l <= target), None)
    curve = {p: [[round(t, 3), l] for t, l in list(zip(v["ms"], v["loss"]))[:: max(1, len(v["ms"]) // 15)]]
             for p, v in runs.items()}
    for v in runs.values():
        del v["ms"], v["loss"]
    out["gcp_poisson"] = {"workload": c["desc"] + (f" (nnz scaled to {nnz})" if scale != 1.0 else ""),
                          "runs": runs, "loss_vs_ms": curve,
                          "loss_gap_bf16_vs_fp32": abs(b16["loss_final"] - f32["loss_final"]) / abs(f32["loss_final"]),
                          "ms_bf16_to_fp32_final_loss": t_b16,
                          "speedup_ms_per_iter_bf16_vs_fp32": f32["ms_per_iter"] / b16["ms_per_iter"]}
    return out


def host_workload_stats(inds, dims, order):
    """Rows touched per mode, leaf fibers (distinct prefixes of all levels but
    the leaf, no split) and, in 4-D, distinct level-0/1 prefixes, from host
    index arrays (numpy)."""
    import numpy as np
    rows = [int(np.count_nonzero(np.bincount(i, minlength=d))) for i, d in zip(inds, dims)]
    key = inds[order[0]].astype(np.int64)
    nfbrs = 0
    for li, q in enumerate(order[1:len(order) - 1]):
        key = key * dims[q] + inds[q].astype(np.int64)
        if len(order) == 4 and li == 0:
            nfbrs = int(np.unique(key).size)
    return rows, int(np.unique(key).size), nfbrs


def reference_arm(a, W, config):
    """--impl reference: the reference's own MTTKRP_COO_CPU (oracle/_ref) over
    every nonzero of the workload on all host threads, each step timed whole.
    The tensor comes from the host restatement of the seeded generator
    (oracle/generate.c, bit-identical to the library's), so nothing of this
    repository's CUDA library is loaded."""
    from oracle import oracle as O
    dims, nd = W["dims"], len(W["dims"])
    nnz = a.nnz or W["nnz"]
    R = a.rank or W["R"]
    esz = 4
    T = host_threads()
    t0 = time.perf_counter()
    inds, vals = O.generate(dims, nnz, W["dist"], W["zipf"], W["val"], a.seed, threads=T)
    gen_s = time.perf_counter() - t0
    order = O.order_modes(dims, 2 if nd == 3 else 0)
    rows, nfib, nfbrs = host_workload_stats(inds, dims, order)
    sb = struct_bytes(nd, nnz, nfib, nfbrs)
    step_bytes = sum(mode_bytes(nd, dims, m, R, esz, sb, rows) for m in range(nd))
    ref = RefCpuMttkrp(inds, vals, dims, R, T)
    del inds, vals
    times = []
    for i in range(a.warmup + a.steps):
        t = ref.seconds()
        if i >= a.warmup:
            times.append(t)
    ts = statistics.mean(times)
    val = step_bytes / ts / 1e9
    line = {"metric": METRIC, "value": val, "unit": "GB/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ts * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, host restatement)",
            "impl": "reference", "config": config,
            "cpu_baseline": {"value": val, "unit": "GB/s", "cores": ref.T, "nproc": T, "kind": ref.kind,
                             "ms_per_step": ts * 1e3,
                             "sample": f"all {nnz} nonzeros, all {nd} modes, every step: MTTKRP_COO_CPU (serial as "
                                       f"shipped, src/mttkrp_cpu.cpp:79) on {ref.T} of {T} host threads over "
                                       f"contiguous nonzero ranges, private outputs added in the step; no "
                                       f"extrapolation"},
            "e2e": {"value": val, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "generate_s": gen_s}
    print(json.dumps(line), flush=True)


def unit_bytes_for(F, nd, dims, nnz, R, esz, rows, plan, info, modes, per_mode):
    """Algorithmic bytes of one launch: a single mode's traversal bytes, or
    for the two-output walk the vals, leaf and middle indices per nonzero,
    slice offsets and indices, every touched row of all factors once, and
    both outputs written once."""
    if len(modes) == 1:
        return per_mode[modes[0]]
    return (nnz * (12 if nd == 3 else 16) + info["n_slices"] * 8 + sum(rows[q] * R * esz for q in range(nd))
            + sum(dims[q] * R * 4 for q in modes))


def per_mode_bytes(F, nd, dims, nnz, R, esz, rows, plan, info):
    """Algorithmic bytes of each mode's MTTKRP under the traversal and kernel
    the plan runs for it."""
    out = []
    for m in range(nd):
        trav = plan[m]["traversal"] if plan else (2 if F.info(4 + m)["present"] else 1)
        pi = F.info(4 + m) if trav == 2 else info
        lvl = pi["mode_order"].index(m)
        k = plan[m].get("kernel") if plan else 0
        if (k == 3 and (nd == 3 or lvl in (0, nd - 1))) or (nd == 3 and k in (4, 5, 6, 7) and lvl == 0) \
                or (nd == 3 and k == 5):
            sb = nnz * (12 if nd == 3 else 16) + pi["n_slices"] * 8  # per-nonzero walks (vals, leaf, mid)
        else:
            sb = struct_bytes(nd, nnz, pi["n_fibers"], pi["n_fbrs"])
        out.append(mode_bytes(nd, dims, m, R, esz, sb, rows))
    return out


# kernel names by mmcsf_kernel_cfg.kernel: one mode, and the two-output walk
SINGLE_KERNELS = {1: "k_mttkrp", 2: "k_mttkrp_flat", 3: "k_mttkrp_rows", 4: "k_mttkrp_fib", 5: "k_mttkrp_rowsv",
                  6: "k_mttkrp_il", 7: "k_mttkrp_stg"}
PAIR_KERNELS = {0: "k_mttkrp_pair", 2: "k_mttkrp_flat", 3: "k_mttkrp_pair", 4: "k_mttkrp_fib", 5: "k_mttkrp_pairv",
                6: "k_mttkrp_il", 7: "k_mttkrp_stg"}


def kernel_label(F, nd, plan, info, modes):
    """(kernel name, description) of one launch of the step."""
    if len(modes) == 2:
        pk = plan.get("pair", {}).get("kernel", 0) if plan else 0
        k = PAIR_KERNELS.get(pk, "k_mttkrp_pair") if nd == 3 else "k_mttkrp_pair4"
        return k, (f"{k} modes {modes[0]} and {modes[1]} (levels 0 and 1 of order {info['mode_order']}, "
                   f"MM-CSF partition, one walk)")
    dom = modes[0]
    trav = plan[dom]["traversal"] if plan else 1
    order = F.info(4 + dom)["mode_order"] if trav == 2 else info["mode_order"]
    lvl = order.index(dom)
    k = plan[dom].get("kernel", 0) if plan else 0
    k = k or (2 if nd == 3 else 1)
    if nd == 3 and k == 7 and lvl != 0:
        k = 6  # the staged walk covers the 3-D slice level (R 16..128, every rank this benchmark runs)
    if nd == 3 and k in (4, 6) and lvl != 0:
        k = 5 if k == 6 else 3
    if nd == 4 and k in (4, 5, 6, 7):
        k = 3
    if k == 3 and nd == 4 and lvl not in (0, 3):
        k = 1  # the 4-D middle levels run the per-team fiber walk
    name = SINGLE_KERNELS[k]
    return name, f"{name} mode {dom} (level {lvl} of order {order}, {'view' if trav == 2 else 'MM-CSF partition'})"


def run_step(F, nd, dims, nnz, R, U, outs, plan, steps, warmup, info, rows, hbm_peak, peak_kind, workload, dtype,
             stream=None):
    """Time the all-mode step launch by launch; returns the per-launch report
    and the dominant launch's roofline entry."""
    import torch
    esz = U[0].element_size()
    stream = stream or torch.cuda.current_stream()
    per_mode = per_mode_bytes(F, nd, dims, nnz, R, esz, rows, plan, info)
    units = step_units(F, U, outs, plan)
    for _ in range(warmup):
        F.mttkrp_all(U, outs)
    launches = F.last_launches
    unit_ms, total_ms = time_units(units, steps, stream)
    ub = [unit_bytes_for(F, nd, dims, nnz, R, esz, rows, plan, info, u[0], per_mode) for u in units]
    di = max(range(len(units)), key=lambda i: unit_ms[i])
    dk, dlabel = kernel_label(F, nd, plan, info, units[di][0])
    achieved = ub[di] / (unit_ms[di] / 1e3) / 1e9
    traffic = traffic_from_profiles(workload, R, dtype, "".join(str(m) for m in units[di][0]), dk)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)", "kernel": dlabel,
                "algorithmic_bytes": ub[di], "avg_ms": unit_ms[di]}
    report = [{"modes": list(u[0]), "kernel": kernel_label(F, nd, plan, info, u[0])[0], "ms": t,
               "algorithmic_bytes": b, "roofline_frac": b / (t / 1e3) / 1e9 / hbm_peak}
              for u, t, b in zip(units, unit_ms, ub)]
    return {"total_ms": total_ms, "ms_per_step": total_ms / steps, "units": report, "roofline": roofline,
            "launches_per_step": launches, "dominant": (di, units[di][0], dk)}


def fp64_refs(inds_dev, vals_dev, U):
    return [fp64_mttkrp(inds_dev, vals_dev, U, m) for m in range(len(U))]


def r64_section(F, X, dims, rows, nfib, info, steps, warmup, hbm_peak, peak_kind, workload):
    """The metric's workload at R = 64 (its second rank): the same format,
    FP32 and BF16 factors, each tuned; step time, the dominant launch's
    roofline fraction and the FP64 errors. The reference's kernels are only
    correct up to R = 32 (src/mttkrp_gpu.cu:746-753), so only the oracle
    checks this rank."""
    import torch
    nd, nnz, R = len(dims), X.nnz, 64
    g = torch.Generator(device="cuda").manual_seed(4321)
    U = [torch.rand(d, R, device="cuda", generator=g) for d in dims]
    outs = [torch.empty(d, R, device="cuda") for d in dims]
    inds_dev, vals_dev = X.device_tensors()
    sb = struct_bytes(nd, nnz, nfib, info["n_fbrs"] if nd == 4 else 0)
    res = {}
    for name, UU in (("f32", U), ("bf16", [u.to(torch.bfloat16) for u in U])):
        plan = F.tune(UU, outs)
        r = run_step(F, nd, dims, nnz, R, UU, outs, plan, steps, warmup, info, rows, hbm_peak, peak_kind,
                     workload, name)
        F.mttkrp_all(UU, outs)
        torch.cuda.synchronize()
        esz = UU[0].element_size()
        step_bytes = sum(mode_bytes(nd, dims, m, R, esz, sb, rows) for m in range(nd))
        errs = []
        for m in range(nd):
            ref = fp64_mttkrp(inds_dev, vals_dev, UU, m)
            errs.append(err_vs(outs[m], ref))
            del ref
        res[name] = {"ms_per_step": r["ms_per_step"], "value_gbs": step_bytes / (r["ms_per_step"] / 1e3) / 1e9,
                     "units": r["units"], "roofline_frac": r["roofline"]["frac"], "dominant": r["roofline"]["kernel"],
                     "plan": plan, "error_vs_fp64": errs}
    return res


def config1_section(steps, warmup, hbm_peak):
    """1000 x 1000 x 1000, 100,000 uniform nonzeros, R = 32, -f 128, -w 1:
    MM-CSF mode 0 and all modes on the device (the reference's -w 1 mapped
    to the worker chunk, and tuned), the library's host COO MTTKRP (-t 1) on
    one thread and all threads, the reference's MTTKRP_COO_CPU on one
    thread, and errors against the FP64 oracle."""
    import numpy as np
    import torch
    import mmcsf
    from oracle import oracle as O
    W = WORKLOADS["uniform3d"]
    dims, nnz, R = W["dims"], W["nnz"], 32
    X = mmcsf.CooTensor.generate(dims, nnz, dist=W["dist"], val_dist=W["val"], seed=0)
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=128, views=1)
    g = torch.Generator(device="cuda").manual_seed(77)
    U = [torch.rand(d, R, device="cuda", generator=g) for d in dims]
    outs = [torch.empty(d, R, device="cuda") for d in dims]
    inds_dev, vals_dev = X.device_tensors()
    refs = fp64_refs(inds_dev, vals_dev, U)
    chunk = F.chunk_for_warps(1, R)
    cfg = mmcsf.KernelCfg()
    cfg.chunk = chunk

    def timed(fn, n):
        for _ in range(warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {"workload": W["desc"] + ", -f 128, -w 1", "chunk_for_w1": chunk}
    out["mode0_w1_ms"] = timed(lambda: F.mttkrp(0, U, outs[0], cfg=cfg), steps)
    e_w1 = err_vs(outs[0], refs[0])
    plan = F.tune(U, outs)
    out["mode0_tuned_ms"] = timed(lambda: F.mttkrp(0, U, outs[0]), steps)
    out["all_modes_tuned_ms"] = timed(lambda: F.mttkrp_all(U, outs), steps)
    F.mttkrp_all(U, outs)
    torch.cuda.synchronize()
    out["error_vs_fp64"] = {"mode0_w1": e_w1, "all_modes_tuned": [err_vs(o, r) for o, r in zip(outs, refs)]}
    out["plan"] = plan
    # host paths: the library's -t 1 and the reference's MTTKRP_COO_CPU
    inds_h, vals_h = X.host_arrays()
    Uh = [u.cpu().numpy() for u in U]
    for name, th in (("host_coo_1thread_ms", 1), ("host_coo_all_threads_ms", 0)):
        o = np.zeros((dims[0], R), np.float32)
        t0 = time.perf_counter()
        for _ in range(5):
            o[:] = 0
            X.mttkrp_host(0, Uh, o, threads=th)
        out[name] = (time.perf_counter() - t0) / 5 * 1e3
    out["error_vs_fp64"]["host_coo_mode0"] = err_vs(torch.from_numpy(o).cuda(), refs[0])
    ref = RefCpuMttkrp(inds_h, vals_h, dims, R, 1)
    t0 = time.perf_counter()
    for _ in range(5):
        ref._run(0, 0)
    out["reference_coo_cpu_mode0_ms"] = (time.perf_counter() - t0) / 5 * 1e3
    out["reference_kind"] = ref.kind
    del F, X
    torch.cuda.empty_cache()
    return out


def skewed4d_section(steps, warmup, seed, hbm_peak, peak_kind):
    """The 4-D workload (1,000,000 x 20,000 x 5,000 x 200, 140M nonzeros, R =
    32): MM-CSF over all modes (views for every mode, tuned, the 4-D
    two-output walk when it wins) against B-CSF (-t 8) and HB-CSF (-t 10) for
    every mode, FP32 factors, with roofline fractions and FP64 errors; and
    the MM-CSF step with BF16 factors."""
    import torch
    import mmcsf
    W = WORKLOADS["skewed4d"]
    dims, nnz, R, nd = W["dims"], W["nnz"], W["R"], 4
    X = mmcsf.CooTensor.generate(dims, nnz, dist=W["dist"], zipf_s=W["zipf"], val_dist=W["val"], seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, views=2)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    info = F.info(2)
    inds_dev, vals_dev = device_coo(X)
    rows, nfib = workload_stats(inds_dev, dims, info["mode_order"])
    g = torch.Generator(device="cuda").manual_seed(99)
    U = [torch.rand(d, R, device="cuda", generator=g) for d in dims]
    outs = [torch.empty(d, R, device="cuda") for d in dims]
    plan = F.tune(U, outs)
    r = run_step(F, nd, dims, nnz, R, U, outs, plan, steps, warmup, info, rows, hbm_peak, peak_kind, "skewed4d", "f32")
    F.mttkrp_all(U, outs)
    torch.cuda.synchronize()
    refs = fp64_refs(inds_dev, vals_dev, U)
    sb = struct_bytes(nd, nnz, nfib, info["n_fbrs"])
    step_bytes = sum(mode_bytes(nd, dims, m, R, 4, sb, rows) for m in range(nd))
    out = {"workload": W["desc"], "format_build_ms": build_ms,
           "mmcsf": {"ms_per_step": r["ms_per_step"], "value_gbs": step_bytes / (r["ms_per_step"] / 1e3) / 1e9,
                     "units": r["units"], "roofline": r["roofline"], "plan": plan,
                     "error_vs_fp64": [err_vs(o, ref) for o, ref in zip(outs, refs)]}}
    Ub = [u.to(torch.bfloat16) for u in U]
    planb = F.tune(Ub, outs)
    rb = run_step(F, nd, dims, nnz, R, Ub, outs, planb, steps, warmup, info, rows, hbm_peak, peak_kind, "skewed4d",
                  "bf16")
    out["mmcsf_bf16"] = {"ms_per_step": rb["ms_per_step"], "units": rb["units"],
                         "roofline_frac": rb["roofline"]["frac"]}
    del F
    torch.cuda.empty_cache()
    out.update(format_section(X, dims, R, U, rows, hbm_peak, refs))
    del X, inds_dev, vals_dev, refs
    torch.cuda.empty_cache()
    return out


def reference_gpu_section(X, F, dims, R, ours_ms):
    """The reference's own GPU MTTKRP (MTTKRP_MIHCSR_GPU,
    src/mttkrp_gpu.cu:3380-3784, built for sm_100a from its sources as
    oracle/_ref/libmmcsf_ref_gpu.so) on this B200, on the MM-CSF arrays this
    library builds (bit-exact to the reference's builders), at its defaults
    (-w 4 -s 1 -b 128, no split) and at the settings of its own benchmark
    script (scripts/run_all.sh:22-23: -f 128 -w 1 -s 4 -b 128 and -s 16 -b
    512). Its "Total GPU time" (the sum of its per-launch event times,
    src/mttkrp_gpu.cu:3757) beside this library's all-mode step. R <= 32
    only: its kernels are wrong above 32 (src/mttkrp_gpu.cu:746-753)."""
    import numpy as np
    import torch
    import mmcsf
    from oracle import oracle as O
    if not O.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libmmcsf_ref_gpu.so was not built (needs the reference sources)"}
    if R > 32:
        return {"unavailable": "the reference's kernels are correct only for R <= 32"}
    info = F.info(2)
    Uc = [torch.full((d, R), m + 0.5, device="cuda") for m, d in enumerate(dims)]
    mine = F.mttkrp(len(dims) - 1, Uc).cpu().numpy()
    runs = {}
    for w, s_, b, f in ((4, 1, 128, 0), (1, 4, 128, 128), (1, 16, 512, 128)):
        G = F if f == 0 else mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=f)
        arr = dict(fbr_ptr=[G.export(2, "fbrPtr0"), G.export(2, "fbrPtr1")],
                   fbr_idx=[G.export(2, "fbrIdx0"), G.export(2, "fbrIdx1")],
                   fbr_like=G.export(2, "fbrLikeSlcInds"), leaf=G.export(2, "indsLeaf"), vals=G.export_f32(2, "vals"))
        if G is not F:
            del G
        torch.cuda.empty_cache()
        ms, out = O.ref_mihcsr_gpu(dims, R, 2, info["mode_order"], warp_per_slice=w, tb_size=b, fiber_per_warp=s_,
                                   **arr)
        runs[f"-w {w} -s {s_} -b {b} -f {f or 'none'}"] = {
            "total_gpu_ms": ms, "last_mode_max_abs_diff_over_max": float(np.abs(out - mine).max() / np.abs(mine).max())}
        del arr
    best = min(runs.values(), key=lambda r: r["total_gpu_ms"])["total_gpu_ms"]
    return {"what": "MTTKRP_MIHCSR_GPU, all modes, R=32, FP32, the reference's kernels built for sm_100a",
            "runs": runs, "best_total_gpu_ms": best, "ours_ms_per_step": ours_ms, "speedup_vs_best": best / ours_ms}


def autotune_section(X, dims, R, steps, warmup, inds_dev, vals_dev, budget=1e-3):
    """The autotuner over the fiber-split threshold (-f none / 128 / 32, each
    format rebuilt) and the factor precision per mode (BF16 copies of the
    FP32 factors where faster and within `budget` of the FP32-factor
    output): the chosen -f, the per-mode plan, the mixed all-mode step's
    time and its errors against the FP64 oracle of the FP32 factors."""
    import torch
    import mmcsf
    g = torch.Generator(device="cuda").manual_seed(1234)
    U = [torch.rand(d, R, device="cuda", generator=g) for d in dims]
    outs = [torch.empty(d, R, device="cuda") for d in dims]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    F, plan = mmcsf.autotune(X, U, views=1, f_candidates=(0, 128, 32), error_budget=budget, outs=outs)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t0
    for _ in range(warmup):
        F.mttkrp_all(U, outs)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        F.mttkrp_all(U, outs)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    F.mttkrp_all(U, outs)
    torch.cuda.synchronize()
    errs = []
    for m in range(len(dims)):
        ref = fp64_mttkrp(inds_dev, vals_dev, U, m)
        errs.append(err_vs(outs[m], ref))
        del ref
    out = {"error_budget": budget, "f_candidates": [0, 128, 32], "chosen_fiber_threshold": plan["fiber_threshold"],
           "plan": plan, "ms_per_step": ms, "launches_per_step": F.last_launches, "tune_and_build_s": tune_s,
           "error_vs_fp64_fp32_factors": errs}
    del F
    torch.cuda.empty_cache()
    return out


def sharded_arm(a, W, config, world, rank, local):
    """--gpus N > 1 (or --sharded): ONE tensor (the same seeded tensor on
    every rank) with every mode's rows split across the ranks (mmcsf.dist
    ShardedMttkrp: each rank runs, for every mode, the MTTKRP of its owned
    rows on a single-mode CSF of its shard; no exchange in the step). Total
    work is fixed as N grows (strong scaling); value = the workload's
    algorithmic bytes (the single-GPU definition) / the step time, max over
    ranks."""
    import torch
    import torch.distributed as dist
    import mmcsf
    from mmcsf import dist as D
    dims, nd = W["dims"], len(W["dims"])
    nnz = a.nnz or W["nnz"]
    R = a.rank or W["R"]
    hbm_peak, peak_kind = peaks()
    X = mmcsf.CooTensor.generate(dims, nnz, dist=W["dist"], zipf_s=W["zipf"], val_dist=W["val"], seed=a.seed)
    inds_dev, vals_dev = device_coo(X)
    order = [2] + sorted([m for m in range(nd) if m != 2], key=lambda m: (dims[m], m))
    rows, nfib = workload_stats(inds_dev, dims, order)
    step_bytes = sum(mode_bytes(nd, dims, m, R, 4, struct_bytes(nd, nnz, nfib, 0), rows) for m in range(nd))
    del X
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sm = D.ShardedMttkrp(dims, inds_dev, vals_dev, device="cuda")
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    del inds_dev, vals_dev
    torch.cuda.empty_cache()
    g = torch.Generator(device="cuda").manual_seed(1234)
    U = [torch.rand(d, R, device="cuda", generator=g) for d in dims]
    slabs = [torch.empty(max(1, hi - lo), R, device="cuda") for lo, hi in sm.rows]
    sm.tune(U)
    stream = torch.cuda.current_stream()
    units = [((m,), lambda m=m: sm.local(m, U, out=slabs[m][:sm.rows[m][1] - sm.rows[m][0]])) for m in range(nd)]
    for _ in range(a.warmup):
        for _, fn in units:
            fn()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    unit_ms, total_ms = time_units(units, a.steps, stream)
    if world > 1:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    tmax = torch.tensor([total_ms], device="cuda")
    if world > 1:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    total_ms = float(tmax.item())
    ms_per_step = total_ms / a.steps
    value = step_bytes * a.steps / (total_ms / 1e3) / 1e9
    # e2e: every factor up from pinned host memory (the shards read rows of
    # all of them), every owned output slab down, per step
    hU = [u.cpu().pin_memory() for u in U]
    hO = [torch.empty(s_.shape).pin_memory() for s_ in slabs]
    dU = [torch.empty_like(u) for u in U]

    def e2e_step():
        for h, d in zip(hU, dU):
            d.copy_(h, non_blocking=True)
        for m in range(nd):
            lo, hi = sm.rows[m]
            sm.local(m, dU, out=slabs[m][:hi - lo])
            hO[m].copy_(slabs[m], non_blocking=True)
    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ke = max(1, min(a.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    em = torch.tensor([e0.elapsed_time(e1) / ke], device="cuda")
    if world > 1:
        dist.all_reduce(em, op=dist.ReduceOp.MAX)
    e_ms = float(em.item())
    hb = sum(d * R * 4 for d in dims)
    db = sum(s_.numel() * 4 for s_ in slabs)
    shard_info = torch.tensor([float(x) for x in sm.shard_nnz], device="cuda")
    all_info = [torch.zeros_like(shard_info) for _ in range(world)] if world > 1 else [shard_info]
    if world > 1:
        dist.all_gather(all_info, shard_info)
    if rank == 0:
        di = max(range(nd), key=lambda i: unit_ms[i])
        # the dominant launch's share of the workload's bytes: its mode's bytes x the shard's share of nonzeros
        ub = mode_bytes(nd, dims, di, R, 4, struct_bytes(nd, nnz, nfib, 0), rows) * sm.shard_nnz[di] / nnz
        achieved = ub / (unit_ms[di] / 1e3) / 1e9
        line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded device generator)",
                "config": dict(config, parallelism=f"row-sharded x{world}: every mode's rows split across the ranks "
                                                   f"by nonzero count, each rank's MTTKRP writes only its rows (no "
                                                   f"collective in the step)"),
                "format_build_ms": build_ms,
                "units": [{"modes": [m], "ms": t, "rank": 0, "shard_nnz": sm.shard_nnz[m]} for m, t in
                          zip(range(nd), unit_ms)],
                "shard_nnz_per_rank": [[int(x) for x in t.tolist()] for t in all_info],
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                             "frac": achieved / hbm_peak, "traffic": None,
                             "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                             "kernel": f"rank 0, mode {di} on its B-CSF shard (bytes: the mode's share by nonzeros)",
                             "algorithmic_bytes": ub, "avg_ms": unit_ms[di]},
                "cpu_baseline": None,
                "e2e": {"value": step_bytes / (e_ms / 1e3) / 1e9, "unit": "GB/s", "ms_per_step": e_ms,
                        "h2d_bytes_per_step": hb, "d2h_bytes_per_step": db},
                "gpu_launches": nd * a.steps, "clocks": clocks}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    W = WORKLOADS[a.workload]
    if a.views is None:
        a.views = W.get("views", 1)
    dims = W["dims"]
    nd = len(dims)
    nnz = a.nnz or W["nnz"]
    R = a.rank or W["R"]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": a.workload, "desc": W["desc"], "nnz": nnz, "R": R,
              "format": f"MM-CSF (-t 12, -m 0), views={a.views}",
              "fiber_threshold": a.fiber_threshold or "none", "factor_dtype": a.dtype,
              "l2": "inputs larger than L2 (structure > 800 MB per step)", "seed": a.seed,
              "parallelism": "single GPU"}
    if a.impl == "reference":
        if rank == 0:
            reference_arm(a, W, config)
        return

    import torch
    import torch.distributed as dist
    esz = 4 if a.dtype == "f32" else 2
    hbm_peak, peak_kind = peaks()
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    if world > 1 or a.sharded:
        sharded_arm(a, W, config, world, rank, local)
        return
    import mmcsf
    X = mmcsf.CooTensor.generate(dims, nnz, dist=W["dist"], zipf_s=W["zipf"], val_dist=W["val"],
                                 seed=a.seed)
    torch.cuda.synchronize()
    tb0 = time.perf_counter()
    F = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, mode=0, fiber_threshold=a.fiber_threshold, views=a.views)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - tb0) * 1e3  # device construction: sorts, CSF levels, views, tables
    info = F.info(2)
    inds_dev, vals_dev = device_coo(X)
    rows, nfib_nosplit = workload_stats(inds_dev, dims, info["mode_order"])
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    tdt = torch.float32 if a.dtype == "f32" else torch.bfloat16
    U = [torch.rand(d, R, device="cuda", generator=g).to(tdt) for d in dims]
    outs = [torch.empty(d, R, device="cuda") for d in dims]
    if a.plan_file:
        if a.plan_file.lstrip().startswith("{"):
            pj = json.loads(a.plan_file)
        else:
            with open(a.plan_file) as fh:
                pj = json.load(fh)
        plan = {(int(k) if k.isdigit() else k): v for k, v in pj.items()}
        F.set_plan(plan)
    else:
        plan = None if a.no_tune else F.tune(U, outs)
    # value: the workload's bytes under the MM-CSF partition traversal (the
    # same definition the reference arm uses, so the two values compare as
    # times); roofline: the bytes of the traversal each launch actually ran
    sb_part = struct_bytes(nd, nnz, nfib_nosplit, info["n_fbrs"] if nd == 4 else 0)
    step_bytes = sum(mode_bytes(nd, dims, m, R, esz, sb_part, rows) for m in range(nd))
    stream = torch.cuda.current_stream()
    per_mode = per_mode_bytes(F, nd, dims, nnz, R, esz, rows, plan, info)
    units = step_units(F, U, outs, plan)
    for _ in range(a.warmup):
        F.mttkrp_all(U, outs)
    launches_per_step = F.last_launches
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    unit_ms, total_ms = time_units(units, a.steps, stream)
    if world > 1:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    tmax = torch.tensor([total_ms], device="cuda")
    if world > 1:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    total_ms = float(tmax.item())
    ms_per_step = total_ms / a.steps
    value = world * step_bytes * a.steps / (total_ms / 1e3) / 1e9

    # e2e through the host-buffer C-ABI call (pinned host memory)
    e2e = None
    if not a.no_e2e and a.dtype == "f32":
        hU = [u.float().cpu().pin_memory() for u in U]
        hO = [torch.empty(d, R).pin_memory() for d in dims]
        for _ in range(min(a.warmup, 2)):
            F.mttkrp_all_host(hU, hO)
        ke = max(1, min(a.steps, 20))
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ke):
            F.mttkrp_all_host(hU, hO)
        e1.record(stream)
        torch.cuda.synchronize()
        em = torch.tensor([e0.elapsed_time(e1)], device="cuda")
        if world > 1:
            dist.all_reduce(em, op=dist.ReduceOp.MAX)
        e_ms = float(em.item()) / ke
        hb = sum(d * R * 4 for d in dims)
        e2e = {"value": world * step_bytes / (e_ms / 1e3) / 1e9, "unit": "GB/s", "ms_per_step": e_ms,
               "h2d_bytes_per_step": hb, "d2h_bytes_per_step": hb}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    ub = [unit_bytes_for(F, nd, dims, nnz, R, esz, rows, plan, info, u[0], per_mode) for u in units]
    di = max(range(len(units)), key=lambda i: unit_ms[i])
    dk, dlabel = kernel_label(F, nd, plan, info, units[di][0])
    achieved = ub[di] / (unit_ms[di] / 1e3) / 1e9
    traffic = traffic_from_profiles(a.workload, R, a.dtype, "".join(str(m) for m in units[di][0]), dk)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "kernel": dlabel, "algorithmic_bytes": ub[di], "avg_ms": unit_ms[di]}
    unit_report = [{"modes": list(u[0]), "kernel": kernel_label(F, nd, plan, info, u[0])[0], "ms": t,
                    "algorithmic_bytes": b, "roofline_frac": b / (t / 1e3) / 1e9 / hbm_peak}
                   for u, t, b in zip(units, unit_ms, ub)]
    # the outputs of the timed step against the FP64 oracle
    F.mttkrp_all(U, outs)
    torch.cuda.synchronize()
    refs = fp64_refs(inds_dev, vals_dev, U)
    errors = [err_vs(o, r) for o, r in zip(outs, refs)]
    # gather ceiling: the same GPU gathering the leaf factor's rows for the
    # workload's own leaf-mode index stream with nothing else to do
    if a.dtype == "f32" and R in (16, 32, 64, 128):
        import ctypes
        from mmcsf._lib import lib as _mlib, check as _mcheck
        leafm = info["mode_order"][-1]
        pms = ctypes.c_float()
        _mcheck(_mlib().mmcsf_probe_gather(ctypes.c_void_p(inds_dev[leafm].data_ptr()), ctypes.c_uint64(nnz),
                                           ctypes.c_void_p(U[leafm].data_ptr()), ctypes.c_uint64(dims[leafm]), R, 5,
                                           ctypes.byref(pms), ctypes.c_void_p(stream.cuda_stream)))
        roofline["gather_ceiling"] = {
            "ms": pms.value, "rows_per_s": nnz / (pms.value / 1e3),
            "what": f"{nnz} rows of the {dims[leafm]} x {R} FP32 mode-{leafm} factor gathered by the workload's "
                    f"mode-{leafm} indices and summed (mmcsf_probe_gather), nothing else"}
        if R in (16, 32, 64):
            # the same rows landed in shared memory by the copy engine (one bulk copy per row, mbarriers)
            tma = {}
            for st_, w_ in ((4, 8), (8, 6)):
                tms = ctypes.c_float()
                rc = _mlib().mmcsf_probe_gather_tma(ctypes.c_void_p(inds_dev[leafm].data_ptr()), ctypes.c_uint64(nnz),
                                                    ctypes.c_void_p(U[leafm].data_ptr()), ctypes.c_uint64(dims[leafm]),
                                                    R, st_, w_, 3, ctypes.byref(tms), ctypes.c_void_p(stream.cuda_stream))
                tma[f"stages{st_}_warps{w_}"] = tms.value if rc == 0 else None
            roofline["gather_ceiling"]["tma_bulk_copy_ms"] = tma
    cpu = None
    if not a.no_cpu and world == 1:
        inds_h, vals_h = X.host_arrays()
        ref = RefCpuMttkrp(inds_h, vals_h, dims, R, host_threads())
        del inds_h, vals_h
        ref.seconds()  # warm-up (page faults of the private outputs)
        ts = min(ref.seconds() for _ in range(2))
        cpu = {"value": step_bytes / ts / 1e9, "unit": "GB/s", "cores": ref.T, "nproc": host_threads(),
               "kind": ref.kind, "ms_per_step": ts * 1e3,
               "sample": f"all {nnz} nonzeros, all {nd} modes: MTTKRP_COO_CPU on {ref.T} host threads over "
                         f"contiguous nonzero ranges (private outputs added in the step), best of 2 steps after "
                         f"one warm-up; no extrapolation"}
    bf16 = None
    if a.dtype == "f32" and not a.no_bf16:
        F.mttkrp_all(U, outs)
        bf16 = bf16_section(F, U, outs, min(a.steps, 20), a.warmup, inds_dev, vals_dev, refs)
    r64 = None
    if a.workload == "skewed3d" and R == 32 and a.dtype == "f32" and not a.no_r64 and not a.nnz:
        r64 = r64_section(F, X, dims, rows, nfib_nosplit, info, min(a.steps, 20), a.warmup, hbm_peak, peak_kind,
                          a.workload)
    refgpu = None
    if nd == 3 and a.dtype == "f32" and not a.no_refgpu and not a.nnz and a.fiber_threshold == 0:
        refgpu = reference_gpu_section(X, F, dims, R, ms_per_step)
    auto = None
    if a.workload == "skewed3d" and R == 32 and a.dtype == "f32" and not a.no_autotune and not a.nnz:
        auto = autotune_section(X, dims, R, min(a.steps, 20), a.warmup, inds_dev, vals_dev)
    ttm = ttm_section(X, dims, R, info["mode_order"][0], rows) if nd == 3 and R in (4, 8, 16, 32, 64, 128) else None
    heur = None
    if not a.no_heuristic:
        heur = heuristic_section(X, dims, R, tdt, a.views)
    formats = None
    if nd == 4 and not a.no_formats:
        fm = format_section(X, dims, R, U, rows, hbm_peak, refs)
        fm["mmcsf"] = {"all_mode_ms": ms_per_step}
        formats = fm
    del refs
    del F, X, U, outs, inds_dev, vals_dev
    torch.cuda.empty_cache()
    cfg1 = None
    if not a.no_config1 and a.workload == "skewed3d" and not a.nnz:
        cfg1 = config1_section(min(a.steps, 20), a.warmup, hbm_peak)
    w4d = None
    if not a.no_4d and a.workload == "skewed3d" and not a.nnz:
        w4d = skewed4d_section(min(a.steps, 10), a.warmup, a.seed, hbm_peak, peak_kind)
    cp = None
    if not a.no_cp:
        cp = cp_section(a.seed, a.cp_scale)
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": a.dtype, "data": "synthetic (seeded device generator)",
            "config": config, "format_build_ms": build_ms, "units": unit_report, "plan": plan, "format": info,
            "roofline": roofline, "error_vs_fp64": errors,
            "cpu_baseline": cpu,
            "e2e": e2e, "gpu_launches": launches_per_step * a.steps, "clocks": clocks, "bf16_factors": bf16,
            "reference_gpu": refgpu, "r64": r64, "autotune": auto, "config1": cfg1, "skewed4d": w4d,
            "ttm": ttm, "cp": cp, "formats": formats, "partition_heuristic": heur}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
