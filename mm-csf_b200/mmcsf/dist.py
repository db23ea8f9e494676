"""One tensor over several GPUs: one process per GPU, torch.distributed for the
exchange (NCCL on GPUs).

The reference has only a sketch of this (src/mttkrp_mpi.h:75-173, not built
by its Makefile): the slices of one mode are split across ranks so that every
rank gets about the same number of nonzeros. Here every mode is split that
way, and each rank owns rows in every mode:

* shard_slices: rank r owns the contiguous row range [b_r, b_{r+1}) of a mode
  holding about nnz / world of its nonzeros (the reference sketch's
  balancing rule), for every mode separately;
* ShardedMttkrp: for every mode m, each rank keeps the nonzeros whose mode-m
  index falls in its range as a single-mode CSF of mode m (the reference's
  mode-m order, order_tensormode), with the mode-m index rebased to the range.
  MTTKRP of mode m on a rank then writes exactly its owned rows: no
  reduction and no exchange. A rank stores about nd * nnz / world nonzeros,
  what a single GPU stores for a format with a view of every mode;
* dist_cp_als: CP-ALS over the shards. Per mode update each rank solves its
  owned rows against the replicated R x R Hadamard of the Gram matrices; the
  exchange is one all-gather of the updated factor rows (every rank's shards
  read arbitrary rows of the other modes), plus all-reduces of R x R Grams
  and R-vectors (column norms or maxima, the fit's inner product). The update
  rules are those of mmcsf_cpd / the reference's cpd (src/cpd_cpu.cu:484-691)
  with the two fixes the single-GPU path makes (full symmetric Gram product
  in the fit, true column max-norm).

The per-rank compute is the CUDA library (mmcsf.Format, B-CSF of the mode);
`local_mttkrp(sm, mode, factors)` lets host-only callers substitute their own
function returning the owned rows.
"""
import numpy as np
import torch
import torch.distributed as dist

__all__ = ["shard_slices", "ShardedMttkrp", "dist_cp_als"]


def shard_slices(counts, world):
    """Row-range boundaries [b_0 = 0, b_1, ..., b_world = len(counts)]:
    rank r owns rows [b_r, b_{r+1}), about sum(counts) / world nonzeros each
    (a boundary is the first row whose prefix count reaches the target)."""
    counts = np.asarray(counts, np.int64)
    pre = np.cumsum(counts)
    total = int(pre[-1]) if len(pre) else 0
    b = [0]
    for r in range(1, world):
        target = (total * r + world - 1) // world
        b.append(max(b[-1], int(np.searchsorted(pre, target, side="left")) + 1 if total else 0))
    b.append(len(counts))
    return [min(x, len(counts)) for x in b]


def _world_rank(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


class ShardedMttkrp:
    """All-mode MTTKRP of one tensor, every mode's rows split across ranks.

    inds / vals: the WHOLE tensor (numpy, or torch tensors on this rank's
    device: then the shards are selected on the device), identical on every
    rank. rows[m] = (lo, hi): this rank's rows of mode m."""

    def __init__(self, dims, inds, vals, group=None, local_mttkrp=None, device=None):
        self.dims = [int(d) for d in dims]
        self.nd = len(dims)
        self.group = group
        self.world, self.rank = _world_rank(group)
        self.device = device
        self._local = local_mttkrp
        on_dev = isinstance(vals, torch.Tensor)
        self.rows, self.shard_nnz, self.fmts, self.shards = [], [], [], []
        for m in range(self.nd):
            im = inds[m]
            if on_dev:
                counts = torch.bincount(im.long(), minlength=self.dims[m]).cpu().numpy()
            else:
                counts = np.bincount(np.asarray(im, np.int64), minlength=self.dims[m])
            b = shard_slices(counts, self.world)
            lo, hi = b[self.rank], b[self.rank + 1]
            self.rows.append((lo, hi))
            if on_dev:
                sel = (im >= lo) & (im < hi)
                si = [i[sel] for i in inds]
                si[m] = si[m] - lo
                sv = vals[sel]
            else:
                ia = np.asarray(im, np.int64)
                sel = (ia >= lo) & (ia < hi)
                si = [np.asarray(i)[sel] for i in inds]
                si[m] = si[m] - lo
                sv = np.asarray(vals)[sel]
            n = int(sv.shape[0])
            self.shard_nnz.append(n)
            self.shards.append((si, sv))
            fmt = None
            if local_mttkrp is None and n > 0:
                import mmcsf
                sd = list(self.dims)
                sd[m] = max(1, hi - lo)
                if on_dev:
                    X = mmcsf.CooTensor.from_device(sd, [i.int() for i in si], sv.float())
                else:
                    X = mmcsf.CooTensor.from_arrays(sd, [i.astype(np.uint32) for i in si], sv.astype(np.float32))
                fmt = mmcsf.Format(X, impl=mmcsf.IMPL_BCSF, mode=m)
                del X
            self.fmts.append(fmt)
        self.nnz = sum(self.shard_nnz)

    def owned(self, mode):
        return self.rows[mode]

    def tune(self, factors):
        """Tune every mode's shard format on this rank (mmcsf_tune)."""
        for m, f in enumerate(self.fmts):
            if f is not None:
                lo, hi = self.rows[m]
                o = torch.empty((max(1, hi - lo), factors[0].shape[1]), dtype=torch.float32,
                                device=factors[0].device)
                f.tune(self._factors_for(m, factors, hi - lo), [o] * self.nd)

    def _factors_for(self, m, factors, nrows):
        # the mode's own factor is not read by its MTTKRP; any tensor of the right dtype stands in
        return [factors[q] if q != m else factors[q][:max(1, nrows)] for q in range(self.nd)]

    def local(self, mode, factors, out=None):
        """This rank's rows of mode `mode`: a (hi - lo) x R float32 tensor."""
        lo, hi = self.rows[mode]
        R = factors[0].shape[1]
        if self._local is not None:
            return self._local(self, mode, factors)
        if out is None:
            out = torch.empty((hi - lo, R), dtype=torch.float32, device=factors[0].device)
        if self.fmts[mode] is None or hi == lo:
            out.zero_()
            return out
        return self.fmts[mode].mttkrp(mode, self._factors_for(mode, factors, hi - lo), out)

    def gather(self, mode, part):
        """All ranks' rows of a mode assembled into one dims[mode] x R tensor
        (one all-gather; slabs padded to the largest)."""
        if self.world == 1:
            return part
        R = part.shape[1]
        lens = torch.tensor([part.shape[0]], device=part.device)
        all_lens = [torch.zeros_like(lens) for _ in range(self.world)]
        dist.all_gather(all_lens, lens, group=self.group)
        sizes = [int(x) for x in all_lens]
        mx = max(sizes)
        pad = torch.zeros((mx, R), dtype=part.dtype, device=part.device)
        pad[:part.shape[0]] = part
        bufs = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(bufs, pad, group=self.group)
        return torch.cat([b[:s] for b, s in zip(bufs, sizes)], 0)

    def mttkrp(self, mode, factors, gather=True):
        """Mode `mode`: the full dims[mode] x R output (gather=True, one
        all-gather of the owned rows) or only this rank's rows."""
        part = self.local(mode, factors)
        return self.gather(mode, part) if gather else part

    def mttkrp_all(self, factors, gather=True):
        return [self.mttkrp(m, factors, gather) for m in range(self.nd)]

    def xnormsq(self):
        """||X||^2 over all ranks (each nonzero counted once: mode 0's shards
        partition the nonzeros)."""
        v = self.shards[0][1]
        s = float((v.double() ** 2).sum()) if isinstance(v, torch.Tensor) else float(
            np.sum(np.asarray(v, np.float64) ** 2))
        t = torch.tensor([s], dtype=torch.float64, device=self.device or "cpu")
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return float(t.item())

    def allreduce(self, t, op=None):
        if self.world > 1:
            dist.all_reduce(t, op=op or dist.ReduceOp.SUM, group=self.group)
        return t


def dist_cp_als(sm, init, max_iters=10, tol=1e-5):
    """CP-ALS over a ShardedMttkrp. init: list of dims[m] x R float32 tensors
    (identical on every rank, on the compute device). Returns (factors,
    lambda (float64 numpy), fit, history); every rank returns the same."""
    nd = sm.nd
    U = [t.detach().clone().float().contiguous() for t in init]
    R = U[0].shape[1]

    def gram(m):  # Gram of mode m's factor from the owned rows, summed over ranks
        lo, hi = sm.owned(m)
        a = U[m][lo:hi].double()
        return sm.allreduce(a.T @ a)

    ata = [gram(m) for m in range(nd)]
    xn = sm.xnormsq()
    lam = torch.ones(R, dtype=torch.float64, device=U[0].device)
    oldfit, fit, hist = 0.0, 0.0, []
    for it in range(max_iters):
        inner = 0.0
        for m in range(nd):
            lo, hi = sm.owned(m)
            M = sm.local(m, U).double()
            V = torch.ones((R, R), dtype=torch.float64, device=M.device)
            for p in range(nd):
                if p != m:
                    V = V * ata[p]
            L, info = torch.linalg.cholesky_ex(V)
            if int(info) == 0:
                A = torch.cholesky_solve(M.T, L).T
            else:
                A = torch.linalg.solve(V, M.T).T
            if it == 0:
                sq = sm.allreduce((A * A).sum(0))
                lam = torch.sqrt(sq)
                lam = torch.where(lam > 0, lam, torch.ones_like(lam))
            else:
                mx = A.max(0).values if A.shape[0] else torch.full((R,), -torch.inf, dtype=A.dtype, device=A.device)
                lam = torch.clamp(sm.allreduce(mx, dist.ReduceOp.MAX), min=1.0)
            A = A / lam
            U[m] = sm.gather(m, A.float().contiguous())
            ata[m] = gram(m)
            if m == nd - 1:  # the fit's <X, model>: the last mode's owned rows
                inner = float(sm.allreduce((lam * (U[m][lo:hi].double() * M).sum(0)).sum().reshape(1)))
        H = torch.ones((R, R), dtype=torch.float64, device=lam.device)
        for p in range(nd):
            H = H * ata[p]
        norm_mats = abs(float(lam @ H @ lam))
        res = xn + norm_mats - 2 * inner
        if res > 0:
            res = res ** 0.5
        fit = 1 - res / xn ** 0.5
        hist.append(fit)
        if it > 0 and abs(fit - oldfit) < tol:
            break
        oldfit = fit
    lam = lam.clone()
    for m in range(nd):
        n = torch.sqrt((U[m].double() ** 2).sum(0))
        n = torch.where(n > 0, n, torch.ones_like(n))
        lam = lam * n
        U[m] = (U[m].double() / n).float()
    return U, lam.cpu().numpy(), fit, hist
