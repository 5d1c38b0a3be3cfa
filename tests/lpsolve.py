"""FP64 LP oracle for the objective checks: scipy's HiGHS on the CPU.

The reference names HPR-LP on the unreduced model as its objective oracle;
HiGHS (a different solver, same optimum) stands in for it at the sizes the
CPU test-suite uses.  Returns x, the row duals y and reduced costs z in the
convention c - A^T y - z = 0.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.optimize import linprog


def solve(m, n, ptr, idx, val, c, AL, AU, l, u):
    A = sp.csr_matrix((val, idx, ptr), shape=(m, n))
    eq = AL == AU
    ub = ~eq & np.isfinite(AU)
    lb = ~eq & np.isfinite(AL)
    A_ub = sp.vstack([A[ub], -A[lb]]).tocsr()
    b_ub = np.concatenate([AU[ub], -AL[lb]])
    bounds = list(zip(np.where(np.isfinite(l), l, None), np.where(np.isfinite(u), u, None)))
    res = linprog(c, A_ub=A_ub if A_ub.shape[0] else None, b_ub=b_ub if A_ub.shape[0] else None,
                  A_eq=A[eq] if eq.any() else None, b_eq=AL[eq] if eq.any() else None, bounds=bounds,
                  method="highs", options=dict(primal_feasibility_tolerance=1e-10,
                                               dual_feasibility_tolerance=1e-10))
    if res.status != 0:
        return res, None, None
    y = np.zeros(m)
    if A_ub.shape[0]:
        mu = res.ineqlin.marginals
        k = int(ub.sum())
        y[ub] += mu[:k]
        y[lb] -= mu[k:]
    if eq.any():
        y[eq] += res.eqlin.marginals
    z = res.lower.marginals + res.upper.marginals
    return res, y, z


def primal_violation(lp, x):
    A = sp.csr_matrix((lp.values, lp.col_idx, lp.row_ptr), shape=(lp.m, lp.n))
    act = A @ x
    parts = [lp.AL - act, act - lp.AU, lp.l - x, x - lp.u]
    return max(float(np.max(p, initial=-np.inf)) for p in parts)
