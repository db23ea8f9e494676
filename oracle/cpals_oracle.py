"""Test infrastructure, not product code: FP64 restatement of the reference's
CP-ALS (src/cpd_cpu.cu:484-691) used as the precision oracle for mmcsf_cpd.

Same update order and rules as the reference: per iteration and mode, MTTKRP,
solve against the Hadamard of the other Gram matrices (Cholesky, general solve
when not positive definite, src/cpd_cpu.cu:140-208), column 2-norms in the
first iteration and max-norms after (src/cpd_cpu.cu:212-335), Gram update,
then the fit (src/cpd_cpu.cu:442-465) and the |fit - oldfit| < tol stop, and
GetFinalLambda at the end (src/cpd_cpu.cu:406-424). Two reference bugs are
fixed, as in the library: the fit uses the full symmetric Gram product (the
reference reads the unwritten triangle) and the max-norm is a true column
maximum clamped below at 1 (the reference compares against a zeroed lambda).
Only tests/ may import it.
"""
import numpy as np


def mttkrp64(dims, inds, vals, mode, U):
    rows = np.asarray(vals, np.float64)[:, None].copy()
    for q in range(len(dims)):
        if q != mode:
            rows = rows * U[q][np.asarray(inds[q], np.int64)]
    out = np.zeros((dims[mode], U[0].shape[1]), np.float64)
    np.add.at(out, np.asarray(inds[mode], np.int64), rows)
    return out


def cp_als(dims, inds, vals, init, max_iters=10, tol=1e-5):
    nd = len(dims)
    U = [np.asarray(f, np.float64).copy() for f in init]
    R = U[0].shape[1]
    ata = [u.T @ u for u in U]
    xnormsq = float(np.sum(np.asarray(vals, np.float64) ** 2))
    oldfit = 0.0
    history = []
    lam = np.ones(R)
    fit = 0.0
    for it in range(max_iters):
        mlast = None
        for m in range(nd):
            M = mttkrp64(dims, inds, vals, m, U)
            if m == nd - 1:
                mlast = M.copy()
            V = np.ones((R, R))
            for p in range(nd):
                if p != m:
                    V = V * ata[p]
            try:
                L = np.linalg.cholesky(V)
                U[m] = np.linalg.solve(L.T, np.linalg.solve(L, M.T)).T
            except np.linalg.LinAlgError:
                U[m] = np.linalg.solve(V, M.T).T
            if it == 0:
                lam = np.sqrt(np.sum(U[m] ** 2, axis=0))
                lam[~(lam > 0)] = 1.0
            else:
                lam = np.maximum(U[m].max(axis=0), 1.0)
            U[m] = U[m] / lam
            ata[m] = U[m].T @ U[m]
        H = np.ones((R, R))
        for p in range(nd):
            H = H * ata[p]
        norm_mats = abs(float(lam @ H @ lam))
        inner = float(np.sum(lam * np.sum(U[nd - 1] * mlast, axis=0)))
        residual = xnormsq + norm_mats - 2 * inner
        if residual > 0:
            residual = np.sqrt(residual)
        fit = 1 - residual / np.sqrt(xnormsq)
        history.append(fit)
        if it > 0 and abs(fit - oldfit) < tol:
            break
        oldfit = fit
    for m in range(nd):
        n = np.sqrt(np.sum(U[m] ** 2, axis=0))
        n[~(n > 0)] = 1.0
        lam = lam * n
        U[m] = U[m] / n
    return U, lam, fit, history
