"""Gradient-based CP on an MM-CSF format (no counterpart in the reference).

The sampled CP model xhat[x] = sum_r lambda_r prod_m A_m[i_m(x), r] at every
nonzero x runs as one hand-written kernel (mmcsf_sampled_model); its adjoint
with respect to A_n is an MTTKRP of the tensor with the same sparsity and the
upstream gradient as values (mmcsf_cp_adjoint), the same kernels the
reference's MTTKRP_MIHCSR_GPU (src/mttkrp_gpu.cu:3578-3724) stands for. Both
sit behind SampledCP, a torch.autograd.Function, so any loss written in torch
over xhat gets exact factor gradients.

precision="bf16" keeps FP32 master factors for the optimiser, hands the
kernels BF16 copies (half the gather bytes) and returns FP32 gradients
(FP32 accumulation inside the kernels).

poisson_loss is the generalized-CP Poisson loss (f(y, m) = m - y log m) over
ALL entries of the tensor: the sum of the model over every entry is
sum_r lambda_r prod_m colsum(A_m)_r, so only the nonzeros need the sampled
model. gcp_poisson fits nonnegative factors to it with projected Adam and
records the loss against device time.
"""
import time

import torch

__all__ = ["SampledCP", "PoissonNZ", "sampled_cp", "poisson_loss", "gcp_poisson"]


class SampledCP(torch.autograd.Function):
    """xhat = SampledCP.apply(fmt, precision, lam, *factors).

    fmt: mmcsf.Format (MM-CSF, or B-CSF for its built mode's sparsity);
    precision: "fp32" or "bf16" (kernel factor type); lam: rank-R float32
    CUDA tensor or None; factors: dims[m] x R float32 (or bfloat16) CUDA
    tensors. Returns nnz float32 values in the format's nonzero order."""

    @staticmethod
    def forward(ctx, fmt, precision, lam, *factors):
        kdt = torch.bfloat16 if precision == "bf16" else factors[0].dtype
        work = [f.detach().to(kdt).contiguous() for f in factors]
        lam_c = lam.detach().float().contiguous() if lam is not None else None
        out = fmt.sampled_model(work, lam_c)
        ctx.fmt = fmt
        ctx.has_lam = lam is not None
        ctx.dtypes = [f.dtype for f in factors]
        if lam is not None:
            ctx.save_for_backward(lam_c, *work)
        else:
            ctx.save_for_backward(*work)
        return out

    @staticmethod
    def backward(ctx, g):
        saved = ctx.saved_tensors
        lam = saved[0] if ctx.has_lam else None
        work = list(saved[1:] if ctx.has_lam else saved)
        fmt = ctx.fmt
        g = g.detach().float().contiguous()
        nd = len(work)
        grads = [None] * nd
        g_lam = None
        need_lam = ctx.has_lam and ctx.needs_input_grad[2]
        for n in range(nd):
            if not (ctx.needs_input_grad[3 + n] or (n == 0 and need_lam)):
                continue
            if need_lam and n == 0:
                m0 = fmt.cp_adjoint(0, work, g)            # unscaled: lambda applied below
                g_lam = (m0 * work[0].float()).sum(0)
                grads[0] = (m0 * lam).to(ctx.dtypes[0])
            else:
                grads[n] = fmt.cp_adjoint(n, work, g, lam).to(ctx.dtypes[n])
        return (None, None, g_lam, *grads)


class PoissonNZ(torch.autograd.Function):
    """L = PoissonNZ.apply(fmt, precision, eps, *factors) = sum over the
    nonzeros of y log(xhat + eps) (no lambda), through the fused kernel
    (mmcsf_poisson_step): the forward pass also yields w = y / (xhat + eps)
    and the slice mode's gradient, so the backward pass only runs the
    adjoints of the other modes (mmcsf_cp_adjoint with w)."""

    @staticmethod
    def forward(ctx, fmt, precision, eps, *factors):
        kdt = torch.bfloat16 if precision == "bf16" else factors[0].dtype
        work = [f.detach().to(kdt).contiguous() for f in factors]
        w, g_root, loss, root = fmt.poisson_step(work, eps)
        ctx.fmt, ctx.root = fmt, root
        ctx.dtypes = [f.dtype for f in factors]
        ctx.save_for_backward(w, g_root, *work)
        return loss[0].float()

    @staticmethod
    def backward(ctx, go):
        w, g_root, *work = ctx.saved_tensors
        grads = [None] * len(work)
        for n in range(len(work)):
            if not ctx.needs_input_grad[3 + n]:
                continue
            g = g_root if n == ctx.root else ctx.fmt.cp_adjoint(n, work, w)
            grads[n] = (g * go).to(ctx.dtypes[n])
        return (None, None, None, *grads)


def _fused_ok(fmt, factors, lam):
    return (lam is None and fmt.nd == 3 and factors[0].shape[1] in (4, 8, 16, 32, 64)
            and fmt.impl == 12 and len(fmt.partitions()) == 1)


def sampled_cp(fmt, factors, lam=None, precision="fp32"):
    """Differentiable sampled CP model at the format's nonzeros."""
    return SampledCP.apply(fmt, precision, lam, *factors)


def poisson_loss(fmt, factors, y, lam=None, precision="fp32", eps=1e-10, fused=True):
    """sum over every entry of m - y log(m + eps), m the CP model, y the
    tensor (zero off its nonzeros); y: nnz values in the format's order.
    fused: use the one-pass kernel (3-D, no lambda, R <= 64; y must then be
    the format's own values) instead of the sampled model + torch ops."""
    cs = factors[0].float().sum(0)
    for f in factors[1:]:
        cs = cs * f.float().sum(0)
    total = (cs * lam).sum() if lam is not None else cs.sum()
    if fused and _fused_ok(fmt, factors, lam):
        return total - PoissonNZ.apply(fmt, precision, eps, *factors)
    xhat = sampled_cp(fmt, factors, lam, precision)
    return total - (y * torch.log(xhat + eps)).sum()


def gcp_poisson(fmt, rank, iters=100, lr=0.05, precision="fp32", init=None, seed=0, eps=1e-10,
                stop_loss=None, rescale=True, profile=False):
    """Projected-Adam Poisson CP (nonnegative factors, no lambda).

    init: optional list of dims[m] x rank nonnegative FP32 CUDA tensors
    (copied; default uniform [0.25, 0.75)). rescale: scale the initial factors
    so the model's total mass equals the tensor's (sum of y), the usual GCP
    start. lr is relative: Adam's step size is lr times the mean initial
    factor entry, so one setting serves tensors of any size.
    stop_loss: stop once the loss is at or below this value (one host sync
    per iteration; None runs every iteration without host syncs).
    profile: also time the phases of every iteration with CUDA events
    (forward: the fused sampled-model / loss / slice-mode gradient pass and
    the colsum terms; backward: the other modes' adjoints; optimizer: Adam
    and the projection), returned as phase_ms summed over the iterations.
    Returns dict(loss=[...], ms=[...] cumulative device time after each
    iteration, factors, iters, seconds[, phase_ms])."""
    dev = torch.device("cuda")
    g = torch.Generator(device="cpu").manual_seed(seed)
    if init is None:
        init = [torch.rand((d, rank), generator=g).to(dev) * 0.5 + 0.25 for d in fmt.dims]
    masters = [t.detach().clone().float().contiguous() for t in init]
    y = fmt.values()
    if rescale:
        with torch.no_grad():
            cs = masters[0].sum(0)
            for f in masters[1:]:
                cs = cs * f.sum(0)
            ratio = float(y.double().sum()) / max(float(cs.double().sum()), 1e-300)
            k = ratio ** (1.0 / len(masters))
            for f in masters:
                f.mul_(k)
    step = lr * float(torch.cat([f.flatten() for f in masters]).mean())
    for f in masters:
        f.requires_grad_(True)
    opt = torch.optim.Adam(masters, lr=step, fused=True)  # one kernel per step for all factors
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(iters + 1)]
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev[0].record()
    n_done = 0
    pev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(iters)] if profile else None
    for it in range(iters):
        if profile:
            pev[it][0].record()
        opt.zero_grad(set_to_none=True)
        loss = poisson_loss(fmt, masters, y, None, precision, eps)
        if profile:
            pev[it][1].record()
        loss.backward()
        if profile:
            pev[it][2].record()
        opt.step()
        with torch.no_grad():
            for p in masters:
                p.clamp_(min=0.0)
        if profile:
            pev[it][3].record()
        losses.append(loss.detach())
        ev[it + 1].record()
        n_done = it + 1
        if stop_loss is not None and loss.item() <= stop_loss:
            break
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    ms = [ev[0].elapsed_time(ev[i + 1]) for i in range(n_done)]
    out = {"loss": [float(v) for v in torch.stack(losses).cpu()], "ms": ms, "iters": n_done, "seconds": secs,
           "factors": [p.detach() for p in masters], "step": step}
    if profile:
        names = ("forward", "backward", "optimizer")
        out["phase_ms"] = {n: sum(pev[i][k].elapsed_time(pev[i][k + 1]) for i in range(n_done))
                           for k, n in enumerate(names)}
    return out
