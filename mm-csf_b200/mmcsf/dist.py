"""One tensor over several GPUs: one process per GPU, torch.distributed for the
exchange (NCCL on GPUs).

The reference has only a sketch of this (src/mttkrp_mpi.h:75-173, not built
by its Makefile): slices of one mode are split across ranks so that every rank
gets about the same number of nonzeros. Here:

* shard_slices / shard_coo: rank r owns a contiguous range of root-mode slices
  holding about nnz / world nonzeros (the reference sketch's balancing rule);
* ShardedMttkrp: each rank builds its own MM-CSF format over its shard and
  runs every mode's MTTKRP locally. The root mode's output rows are disjoint
  across ranks (no exchange needed for them); every other mode's output is a
  sum over ranks, one all-reduce per mode (full = True also assembles the root
  mode, for callers that need every row on every rank);
* dist_cp_als: CP-ALS over the shards. Per mode update the only exchange is
  the all-reduce of that mode's MTTKRP output; the R x R Gram/Hadamard solve,
  normalisation and fit are replicated (every rank holds identical factors),
  and ||X||^2 is all-reduced once. The update rules are those of
  mmcsf_cpd / the reference's cpd (src/cpd_cpu.cu:484-691) with the two fixes
  the single-GPU path makes (full symmetric Gram product in the fit, true
  column max-norm).

The per-rank compute is the CUDA library (mmcsf.Format); `local_mttkrp` lets
host-only callers substitute their own (mode, factors) -> output function.
"""
import numpy as np
import torch
import torch.distributed as dist

__all__ = ["shard_slices", "shard_coo", "ShardedMttkrp", "dist_cp_als"]


def shard_slices(counts, world):
    """Slice-range boundaries [b_0 = 0, b_1, ..., b_world = len(counts)]:
    rank r owns slices [b_r, b_{r+1}), about sum(counts) / world nonzeros
    each (a boundary is the first slice whose prefix count reaches the
    target)."""
    counts = np.asarray(counts, np.int64)
    pre = np.cumsum(counts)
    total = int(pre[-1]) if len(pre) else 0
    b = [0]
    for r in range(1, world):
        target = (total * r + world - 1) // world
        b.append(max(b[-1], int(np.searchsorted(pre, target, side="left")) + 1 if total else 0))
    b.append(len(counts))
    return [min(x, len(counts)) for x in b]


def shard_coo(dims, inds, vals, world, rank, root_mode):
    """This rank's nonzeros (numpy) and its owned root-mode slice range."""
    root = np.asarray(inds[root_mode], np.int64)
    counts = np.bincount(root, minlength=dims[root_mode])
    b = shard_slices(counts, world)
    lo, hi = b[rank], b[rank + 1]
    sel = (root >= lo) & (root < hi)
    return (lo, hi), [np.asarray(i)[sel] for i in inds], np.asarray(vals)[sel]


def _root_mode(dims):
    """Level-0 mode of the MM-CSF partition the library builds (the
    reference's order for a mode-2 CSF: 2, then the rest by ascending length)."""
    nd = len(dims)
    rest = sorted([m for m in range(nd) if m != 2], key=lambda m: (dims[m], m))
    return 2 if nd >= 3 else rest[0]


class ShardedMttkrp:
    """All-mode MTTKRP of one tensor sharded by root-mode slices."""

    def __init__(self, dims, inds, vals, group=None, root_mode=None, views=1, local_mttkrp=None, device=None):
        self.dims = [int(d) for d in dims]
        self.nd = len(dims)
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.root = _root_mode(self.dims) if root_mode is None else root_mode
        self.rows, self.inds, self.vals = shard_coo(self.dims, inds, vals, self.world, self.rank, self.root)
        self.nnz = len(self.vals)
        self.device = device
        self._local = local_mttkrp
        self.fmt = None
        if local_mttkrp is None and self.nnz > 0:
            import mmcsf
            X = mmcsf.CooTensor.from_arrays(self.dims, [i.astype(np.uint32) for i in self.inds],
                                            self.vals.astype(np.float32))
            self.fmt = mmcsf.Format(X, impl=mmcsf.IMPL_MMCSF, views=views)
            self._coo = X

    def local(self, mode, factors):
        if self._local is not None:
            return self._local(mode, factors)
        if self.nnz == 0:
            return torch.zeros((self.dims[mode], factors[0].shape[1]), dtype=torch.float32,
                               device=factors[0].device)
        return self.fmt.mttkrp(mode, factors)

    def mttkrp(self, mode, factors, full=True):
        """Mode `mode` summed over ranks. full=False leaves the root mode's
        output sharded (only this rank's owned rows are filled)."""
        out = self.local(mode, factors)
        if self.world > 1 and (mode != self.root or full):
            dist.all_reduce(out, op=dist.ReduceOp.SUM, group=self.group)
        return out

    def mttkrp_all(self, factors, full=True):
        return [self.mttkrp(m, factors, full) for m in range(self.nd)]

    def xnormsq(self):
        t = torch.tensor([float(np.sum(np.asarray(self.vals, np.float64) ** 2))], dtype=torch.float64,
                         device=self.device or "cpu")
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return float(t.item())


def dist_cp_als(sm, init, max_iters=10, tol=1e-5):
    """CP-ALS over a ShardedMttkrp. init: list of dims[m] x R float32 tensors
    (identical on every rank, on the compute device). Returns (factors,
    lambda (float64 numpy), fit, history); every rank returns the same."""
    nd = sm.nd
    U = [t.detach().clone().float().contiguous() for t in init]
    R = U[0].shape[1]
    ata = [(u.double().T @ u.double()) for u in U]
    xn = sm.xnormsq()
    lam = torch.ones(R, dtype=torch.float64, device=U[0].device)
    oldfit, fit, hist = 0.0, 0.0, []
    for it in range(max_iters):
        mlast = None
        for m in range(nd):
            M = sm.mttkrp(m, U).double()
            if m == nd - 1:
                mlast = M
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
                lam = torch.sqrt((A * A).sum(0))
                lam = torch.where(lam > 0, lam, torch.ones_like(lam))
            else:
                lam = torch.clamp(A.max(0).values, min=1.0)
            A = A / lam
            U[m] = A.float().contiguous()
            ata[m] = A.T @ A
        H = torch.ones((R, R), dtype=torch.float64, device=lam.device)
        for p in range(nd):
            H = H * ata[p]
        norm_mats = abs(float(lam @ H @ lam))
        inner = float((lam * (U[nd - 1].double() * mlast).sum(0)).sum())
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
