"""Seeded synthetic LP generators for the presolve workloads.

The LPs have the form ``min c'x  s.t.  AL <= A x <= AU,  l <= x <= u`` and are
returned as host CSR arrays (int32 indices, float64 values) plus the CSR of
A^T, matching the device layout of ``LPInfoGpu`` in the reference
(cpp/include/gpu_preprocessor/presolve/presolve_structs.hpp:160-180).

Three families are produced:

* ``random_lp(m, n, seed, hub_rows=0)`` -- the "plain presolve" family: per
  column 1+Poisson(4) nonzeros at uniform rows, values U[-10,10] on a 1e-3 grid,
  with injected singleton rows (5%), two-entry equality rows (5%), scaled copy
  rows (3%), scaled copy columns (2%) and empty columns (2%).  Row sides come
  from a planted point x0 so the LP is feasible.  ``hub_rows`` extra rows get
  log-uniform lengths in [500, 5000] to skew the row-length distribution.
  The 2,000 x 5,000 instance is the CPU-runnable case; 2,000,000 x 5,000,000
  with 2,000 hub rows (~29M nonzeros) is the single-GPU scale case.
* ``qap_lp(N, seed)`` -- the LP relaxation of a quadratic assignment problem in
  Adams-Johnson form, laid out row-for-row and column-for-column like the
  reference's QAP exporter (scripts/generate_qap20.jl:26-112), with flow and
  distance matrices drawn i.i.d. from {0..9} (zero diagonal).

Nothing here reads a benchmark data set; every instance is synthetic.
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

INF = np.inf


@dataclasses.dataclass
class HostLP:
    m: int
    n: int
    row_ptr: np.ndarray   # int32 [m+1]
    col_idx: np.ndarray   # int32 [nnz]
    values: np.ndarray    # float64 [nnz]
    c: np.ndarray
    AL: np.ndarray
    AU: np.ndarray
    l: np.ndarray
    u: np.ndarray
    obj_constant: float = 0.0
    at_ptr: np.ndarray | None = None
    at_idx: np.ndarray | None = None
    at_val: np.ndarray | None = None

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def ensure_transpose(self) -> "HostLP":
        if self.at_ptr is None:
            self.at_ptr, self.at_idx, self.at_val = csr_transpose(
                self.m, self.n, self.row_ptr, self.col_idx, self.values)
        return self


def csr_transpose(m, n, ptr, idx, val):
    """Stable CSR transpose: rows of A^T list the rows of A in ascending order."""
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(ptr))
    order = np.argsort(idx, kind="stable")
    t_idx = rows[order].astype(np.int32)
    t_val = val[order].astype(np.float64)
    counts = np.bincount(idx, minlength=n)
    t_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=t_ptr[1:])
    return t_ptr.astype(np.int32), t_idx, t_val


def _sorted_unique(keys):
    keys = np.sort(keys)
    if keys.size:
        keys = keys[np.concatenate(([True], keys[1:] != keys[:-1]))]
    return keys


def _row_major_order(rows, cols):
    span = int(cols.max()) + 1 if cols.size else 1
    return np.argsort(rows.astype(np.int64) * span + cols, kind="stable")


def coo_to_csr(m, rows, cols, vals):
    order = _row_major_order(rows, cols)
    rows, cols, vals = rows[order], cols[order], vals[order]
    counts = np.bincount(rows, minlength=m)
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    if ptr[-1] > np.iinfo(np.int32).max:
        raise ValueError("nnz exceeds the int32 offset range")
    return ptr.astype(np.int32), cols.astype(np.int32), vals.astype(np.float64)


def _grid_values(rng, k):
    v = np.round(rng.uniform(-10.0, 10.0, size=k), 3)
    bad = v == 0.0
    while bad.any():
        v[bad] = np.round(rng.uniform(-10.0, 10.0, size=int(bad.sum())), 3)
        bad = v == 0.0
    return v


def random_lp(m: int, n: int, seed: int = 0, hub_rows: int = 0, slack_frac: float = 0.0) -> HostLP:
    """Plain-presolve family (see module docstring).  ``slack_frac`` > 0 appends
    one singleton column to that fraction of the rows (see _add_slacks)."""
    rng = np.random.default_rng(seed)
    n_single = int(round(0.05 * m))
    n_dton = int(round(0.05 * m))
    n_copy_rows = int(round(0.03 * m))
    n_normal = m - n_single - n_dton - n_copy_rows
    if n_normal < 1:
        raise ValueError("too few rows")
    # Row roles are interleaved by a permutation so no rule sees a block layout.
    role = np.zeros(m, dtype=np.int8)  # 0 normal, 1 singleton, 2 doubleton eq, 3 copy
    role[n_normal:n_normal + n_single] = 1
    role[n_normal + n_single:n_normal + n_single + n_dton] = 2
    role[n_normal + n_single + n_dton:] = 3
    role = role[rng.permutation(m)]
    normal_rows = np.flatnonzero(role == 0).astype(np.int64)

    n_empty = int(round(0.02 * n))
    n_copy_cols = int(round(0.02 * n))
    crole = np.zeros(n, dtype=np.int8)  # 0 regular, 1 copy, 2 empty
    crole[:n_copy_cols] = 1
    crole[n_copy_cols:n_copy_cols + n_empty] = 2
    crole = crole[rng.permutation(n)]
    regular_cols = np.flatnonzero(crole == 0).astype(np.int64)

    # Regular columns: 1 + Poisson(4) entries at uniformly drawn normal rows.
    per_col = 1 + rng.poisson(4.0, size=regular_cols.size)
    cols = np.repeat(regular_cols, per_col)
    rows = normal_rows[rng.integers(0, normal_rows.size, size=cols.size)]
    key = _sorted_unique(cols * m + rows)       # drop repeated (row, col) draws
    cols, rows = key // m, key % m
    vals = _grid_values(rng, rows.size)

    # Hub rows: extra long rows over regular columns (log-uniform lengths).
    if hub_rows > 0:
        hubs = rng.choice(normal_rows, size=hub_rows, replace=False)
        lengths = np.exp(rng.uniform(np.log(500.0), np.log(5000.0), size=hub_rows)).astype(np.int64)
        lengths = np.minimum(lengths, regular_cols.size)
        h_rows = np.repeat(hubs, lengths)
        h_cols = regular_cols[rng.integers(0, regular_cols.size, size=h_rows.size)]
        base = cols * m + rows
        hkey = _sorted_unique(h_cols * m + h_rows)
        new = hkey[~np.isin(hkey, base, assume_unique=True)]
        new_cols, new_rows = new // m, new % m
        cols = np.concatenate([cols, new_cols])
        rows = np.concatenate([rows, new_rows])
        vals = np.concatenate([vals, _grid_values(rng, new.size)])

    # Copy columns: a regular column scaled by a factor in [0.5, 4] of random sign.
    copy_cols = np.flatnonzero(crole == 1)
    src_cols = regular_cols[rng.integers(0, regular_cols.size, size=copy_cols.size)]
    col_factor = rng.uniform(0.5, 4.0, size=copy_cols.size) * rng.choice([-1.0, 1.0], size=copy_cols.size)
    order = np.argsort(cols, kind="stable")
    cols, rows, vals = cols[order], rows[order], vals[order]
    cstart = np.searchsorted(cols, src_cols, side="left")
    cstop = np.searchsorted(cols, src_cols, side="right")
    lens = cstop - cstart
    take = np.concatenate([np.arange(a, b) for a, b in zip(cstart, cstop)]) if lens.sum() else np.zeros(0, np.int64)
    cc_cols = np.repeat(copy_cols, lens)
    cc_rows = rows[take]
    cc_vals = vals[take] * np.repeat(col_factor, lens)
    cols = np.concatenate([cols, cc_cols])
    rows = np.concatenate([rows, cc_rows])
    vals = np.concatenate([vals, cc_vals])

    # Copy rows: a normal row scaled by U[0.5, 4].
    copy_rows = np.flatnonzero(role == 3)
    src_rows = normal_rows[rng.integers(0, normal_rows.size, size=copy_rows.size)]
    row_factor = rng.uniform(0.5, 4.0, size=copy_rows.size)
    order = _row_major_order(rows, cols)
    cols, rows, vals = cols[order], rows[order], vals[order]
    rstart = np.searchsorted(rows, src_rows, side="left")
    rstop = np.searchsorted(rows, src_rows, side="right")
    rlens = rstop - rstart
    rtake = np.concatenate([np.arange(a, b) for a, b in zip(rstart, rstop)]) if rlens.sum() else np.zeros(0, np.int64)
    cr_rows = np.repeat(copy_rows, rlens)
    cr_cols = cols[rtake]
    cr_vals = vals[rtake] * np.repeat(row_factor, rlens)

    # Singleton rows and two-entry equality rows over regular columns.
    s_rows = np.flatnonzero(role == 1)
    s_cols = regular_cols[rng.integers(0, regular_cols.size, size=s_rows.size)]
    s_vals = _grid_values(rng, s_rows.size)
    d_rows = np.flatnonzero(role == 2)
    d1 = rng.integers(0, regular_cols.size, size=d_rows.size)
    d2 = (d1 + 1 + rng.integers(0, regular_cols.size - 1, size=d_rows.size)) % regular_cols.size
    d_cols = np.stack([regular_cols[d1], regular_cols[d2]], axis=1).reshape(-1)
    d_rows2 = np.repeat(d_rows, 2)
    d_vals = _grid_values(rng, d_rows2.size)

    rows = np.concatenate([rows, cr_rows, s_rows, d_rows2]).astype(np.int64)
    cols = np.concatenate([cols, cr_cols, s_cols, d_cols]).astype(np.int64)
    vals = np.concatenate([vals, cr_vals, s_vals, d_vals]).astype(np.float64)
    ptr, idx, val = coo_to_csr(m, rows, cols, vals)

    # Bounds, planted point, sides and costs.
    l = np.zeros(n)
    u = rng.uniform(1.0, 100.0, size=n)
    inf_u = rng.random(n) < 0.2
    u[inf_u] = INF
    x0 = np.where(inf_u, rng.uniform(0.0, 10.0, size=n), rng.uniform(0.0, 1.0, size=n) * u)
    x0 = np.where(inf_u, x0, np.minimum(x0, u))
    act = np.add.reduceat(val * x0[idx], ptr[:-1]) if idx.size else np.zeros(m)
    act = np.where(np.diff(ptr) > 0, act, 0.0)
    s_lo = rng.uniform(0.0, 5.0, size=m)
    s_hi = rng.uniform(0.0, 5.0, size=m)
    lo_fin = rng.random(m) < 0.5
    hi_fin = rng.random(m) < 0.5
    AL = np.where(lo_fin, act - s_lo, -INF)
    AU = np.where(hi_fin, act + s_hi, INF)
    eq = role == 2
    AL[eq] = act[eq]
    AU[eq] = act[eq]
    c = rng.standard_normal(n)
    c[inf_u] = np.abs(c[inf_u])
    lp = HostLP(m, n, ptr, idx, val, c, AL, AU, l, u)
    if slack_frac > 0.0:
        lp = _add_slacks(lp, act, slack_frac, seed)
    return lp.ensure_transpose()


def _add_slacks(lp: HostLP, act, frac: float, seed: int) -> HostLP:
    """Append one singleton column to a fraction of the rows: nonnegative
    columns, free columns and boxed columns (kinds 0/3, 1, 2).  Half of those
    rows become equalities.  The planted point is extended so the LP stays
    feasible, and the costs of the whole LP are redrawn from a planted dual
    point so it stays bounded."""
    rng = np.random.default_rng(seed + 7919)
    m, n = lp.m, lp.n
    rows = np.flatnonzero(rng.random(m) < frac)
    k = rows.size
    kind = rng.integers(0, 4, size=k)
    coef = _grid_values(rng, k)
    sl = np.where(kind == 1, -INF, 0.0)
    su = np.where(kind == 2, rng.uniform(1.0, 20.0, size=k), INF)
    xs = np.where(kind == 2, rng.uniform(0.0, 1.0, size=k) * su, rng.uniform(0.0, 5.0, size=k))
    shift = coef * xs
    AL, AU = lp.AL.copy(), lp.AU.copy()
    eq = rng.random(k) < 0.5
    eq |= ~np.isfinite(AL[rows]) & ~np.isfinite(AU[rows])   # no slack in a free row
    base = act[rows] + shift
    AL[rows] = np.where(eq, base, AL[rows] + shift)
    AU[rows] = np.where(eq, base, AU[rows] + shift)
    counts = np.diff(lp.row_ptr).astype(np.int64)
    r_all = np.repeat(np.arange(m, dtype=np.int64), counts)
    rows_c = np.concatenate([r_all, rows.astype(np.int64)])
    cols_c = np.concatenate([lp.col_idx.astype(np.int64), n + np.arange(k, dtype=np.int64)])
    vals_c = np.concatenate([lp.values, coef])
    ptr, idx, val = coo_to_csr(m, rows_c, cols_c, vals_c)
    l = np.concatenate([lp.l, sl])
    u = np.concatenate([lp.u, su])
    # Costs from a planted dual point (c = A'y + z with signs that fit the
    # finite sides and bounds), so the LP has a finite optimum even with free
    # columns in it.
    y = np.abs(rng.standard_normal(m)) * (rng.random(m) < 0.5)
    lo_f, hi_f = np.isfinite(AL), np.isfinite(AU)
    y = np.where(lo_f & hi_f, y * rng.choice([-1.0, 1.0], size=m), np.where(lo_f, y, np.where(hi_f, -y, 0.0)))
    zmag = np.abs(rng.standard_normal(n + k)) * (rng.random(n + k) < 0.5)
    l_f, u_f = np.isfinite(l), np.isfinite(u)
    z = np.where(l_f & u_f, zmag * rng.choice([-1.0, 1.0], size=n + k), np.where(l_f, zmag, np.where(u_f, -zmag, 0.0)))
    c = np.zeros(n + k)
    np.add.at(c, idx, val * np.repeat(y, np.diff(ptr)))
    c += z
    return HostLP(m, n + k, ptr, idx, val, c, AL, AU, l, u)


def replicated_lp(m: int, n: int, copies: int, seed: int = 0) -> HostLP:
    """`copies` identical copies of random_lp(m, n) on the block diagonal plus
    one coupling row (sum of all variables <= a slack bound): a model with an
    exact symmetry, so colour refinement folds it back to about one copy."""
    base = random_lp(m, n, seed)
    rows, cols, vals = [], [], []
    counts = np.diff(base.row_ptr).astype(np.int64)
    r_base = np.repeat(np.arange(m, dtype=np.int64), counts)
    for k in range(copies):
        rows.append(r_base + k * m)
        cols.append(base.col_idx.astype(np.int64) + k * n)
        vals.append(base.values)
    mt, nt = m * copies + 1, n * copies
    rows.append(np.full(nt, mt - 1, dtype=np.int64))
    cols.append(np.arange(nt, dtype=np.int64))
    vals.append(np.ones(nt))
    ptr, idx, val = coo_to_csr(mt, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))
    finite_u = np.where(np.isfinite(base.u), base.u, 10.0)
    cap = float(copies * finite_u.sum()) * 2.0 + 1.0
    AL = np.concatenate([np.tile(base.AL, copies), [-INF]])
    AU = np.concatenate([np.tile(base.AU, copies), [cap]])
    return HostLP(mt, nt, ptr, idx, val, np.tile(base.c, copies), AL, AU, np.tile(base.l, copies),
                  np.tile(base.u, copies)).ensure_transpose()


def qap_lp(N: int, seed: int = 0) -> HostLP:
    """Adams-Johnson QAP relaxation in the reference exporter's row/column order."""
    rng = np.random.default_rng(seed)
    flow = rng.integers(0, 10, size=(N, N)).astype(np.float64)
    dist = rng.integers(0, 10, size=(N, N)).astype(np.float64)
    np.fill_diagonal(flow, 0.0)
    np.fill_diagonal(dist, 0.0)
    n2, n3, n4 = N * N, N ** 3, N ** 4
    neq = 2 * N + 2 * n3 + n4
    m = n4 + neq + n2
    n = n2 + n4
    eq0 = n4                      # first equality row
    rng_rows0 = n4 + neq          # first ranged row
    # Zero-based index helpers matching idx2/idx3/idx4 (column-major, 1-based in the exporter).
    i, j = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    i, j = i.reshape(-1), j.reshape(-1)
    xcol = i + N * j
    R, C, V = [], [], []
    t = np.arange(N)
    # x[i,j] column entries.
    R += [eq0 + i, eq0 + N + j]
    C += [xcol, xcol]
    V += [np.ones(n2), np.ones(n2)]
    for tt in range(N):
        R.append(eq0 + 2 * N + (tt + N * i + n2 * j))
        C.append(xcol)
        V.append(-np.ones(n2))
        R.append(eq0 + 2 * N + n3 + (tt + N * i + n2 * j))
        C.append(xcol)
        V.append(-np.ones(n2))
    R.append(rng_rows0 + xcol)
    C.append(xcol)
    V.append(np.ones(n2))
    # y[i,j,k,l] column entries.
    ii, jj, kk, ll = np.meshgrid(t, t, t, t, indexing="ij")
    ii, jj, kk, ll = (a.reshape(-1) for a in (ii, jj, kk, ll))
    q = ii + N * jj + n2 * kk + n3 * ll
    rq = kk + N * ll + n2 * ii + n3 * jj
    ycol = n2 + q
    R += [q, eq0 + 2 * N + (jj + N * kk + n2 * ll), eq0 + 2 * N + n3 + (ii + N * kk + n2 * ll)]
    C += [ycol, ycol, ycol]
    V += [-np.ones(n4), np.ones(n4), np.ones(n4)]
    off = q != rq
    first = np.minimum(q, rq)[off]
    second = np.maximum(q, rq)[off]
    sign = np.where(q < rq, 1.0, -1.0)[off]
    R += [eq0 + 2 * N + 2 * n3 + first, eq0 + 2 * N + 2 * n3 + second]
    C += [ycol[off], ycol[off]]
    V += [sign, -sign]
    rows = np.concatenate(R).astype(np.int64)
    cols = np.concatenate(C).astype(np.int64)
    vals = np.concatenate(V).astype(np.float64)
    ptr, idx, val = coo_to_csr(m, rows, cols, vals)
    c = np.zeros(n)
    c[n2 + q] = flow[ii, kk] * dist[jj, ll]
    AL = np.empty(m)
    AU = np.empty(m)
    AL[:n4], AU[:n4] = -INF, 0.0
    AL[eq0:eq0 + neq] = 0.0
    AU[eq0:eq0 + neq] = 0.0
    AL[eq0:eq0 + 2 * N] = 1.0
    AU[eq0:eq0 + 2 * N] = 1.0
    AL[rng_rows0:], AU[rng_rows0:] = 0.0, 1.0
    l = np.full(n, -INF)
    u = np.full(n, INF)
    return HostLP(m, n, ptr, idx, val, c, AL, AU, l, u).ensure_transpose()


def setcover_lp(m: int, n: int, seed: int = 0, witness: bool = True) -> HostLP:
    """Unit set-covering LP  min c'x, sum_{j in row i} x_j >= 1, 0 <= x <= 1,
    every coefficient 1: the structure the column-domination startup rule
    accepts.  The first max(1, n // 4) columns cost 1 and cover every row
    (column i mod that count is in row i) so each row holds a cost-1
    witness; every column gets 1 + Poisson(2) further distinct rows, and the
    remaining columns an integer cost uniform in [1, 2 * degree], so about
    half of them cost more than their degree.  ``witness=False`` raises the
    cost-1 columns to 2, which leaves rows without a witness."""
    rng = np.random.default_rng(seed)
    cheap = max(1, n // 4)
    rows = [np.arange(m, dtype=np.int64)]
    cols = [np.arange(m, dtype=np.int64) % cheap]
    extra = 1 + rng.poisson(2.0, size=n)
    rows.append(rng.integers(0, m, size=int(extra.sum())))
    cols.append(np.repeat(np.arange(n, dtype=np.int64), extra))
    r, cidx = np.concatenate(rows), np.concatenate(cols)
    key = np.unique(r * n + cidx)                       # distinct (row, column) pairs
    r, cidx = key // n, key % n
    ptr, idx, val = coo_to_csr(m, r, cidx, np.ones(len(r)))
    degree = np.bincount(cidx, minlength=n)
    c = np.floor(rng.uniform(1.0, 2.0 * np.maximum(degree, 1) + 1.0)).astype(np.float64)
    c[:cheap] = 1.0 if witness else 2.0
    AL, AU = np.ones(m), np.full(m, INF)
    return HostLP(m, n, ptr, idx, val, c, AL, AU, np.zeros(n), np.ones(n)).ensure_transpose()


def auxiliary_lp(m: int, n: int, seed: int = 0, pairs: float = 0.02, products: float = 0.02) -> HostLP:
    """random_lp(m, n) plus blocks of new [0, 1] columns and rows that the
    projected-auxiliary Startup rules accept, and decoys they must reject.

    * two-row block (pairs * n of them): a zero-cost t with t >= x/4 and
      t <= 1 - y/4, x and y new columns of nonzero cost;
    * product block (products * n): a zero-cost z with z >= x + y - 1,
      z <= x, z <= y (the McCormick envelope of x y);
    * decoys, one per 16 blocks of each kind: two t sharing their lower row
      (row conflict), a t whose rows leave no margin (t >= x, t <= 1 - y,
      so max(x + y - 1) = 1 > 0), a product whose upper row has
      coefficient -0.5, and a product whose endpoint is itself a product
      variable (endpoint conflict)."""
    base = random_lp(m, n, seed)
    rng = np.random.default_rng(seed + 7919)
    rows, cols, vals = [], [], []
    AL, AU, c = [], [], []
    next_col, next_row = n, m

    def new_cols(k):
        nonlocal next_col
        first = next_col
        next_col += k
        c.extend(np.round(rng.uniform(-3.0, 3.0, size=k), 2).tolist())
        return list(range(first, first + k))

    def new_row(entries, lo, hi):
        nonlocal next_row
        for j, a in entries:
            rows.append(next_row)
            cols.append(j)
            vals.append(a)
        AL.append(lo)
        AU.append(hi)
        next_row += 1

    def two_row(margin=True):
        t, x, y = new_cols(3)
        c[t - n] = 0.0
        q = 0.25 if margin else 1.0
        new_row([(t, 1.0), (x, -q)], 0.0, INF)
        new_row([(t, 1.0), (y, q)], -INF, 1.0)

    def product(upper_coeff=-1.0, endpoint=None):
        z, x, y = new_cols(3)
        c[z - n] = 0.0
        if endpoint is not None:
            x = endpoint
        new_row([(z, 1.0), (x, -1.0), (y, -1.0)], -1.0, INF)
        new_row([(z, 1.0), (x, upper_coeff)], -INF, 0.0)
        new_row([(z, 1.0), (y, -1.0)], -INF, 0.0)
        return z

    for k in range(int(pairs * n)):
        if k % 16 == 5:
            t1, t2, x, y1, y2 = new_cols(5)
            c[t1 - n] = c[t2 - n] = 0.0
            new_row([(t1, 1.0), (t2, 1.0), (x, -0.25)], 0.0, INF)
            new_row([(t1, 1.0), (y1, 0.25)], -INF, 1.0)
            new_row([(t2, 1.0), (y2, 0.25)], -INF, 1.0)
        elif k % 16 == 11:
            two_row(margin=False)
        else:
            two_row()
    for k in range(int(products * n)):
        if k % 16 == 3:
            product(upper_coeff=-0.5)
        elif k % 16 == 9:
            product(endpoint=product())
        else:
            product()
    n_new, m_new = next_col, next_row
    brows = np.repeat(np.arange(m, dtype=np.int64), np.diff(base.row_ptr))
    ptr, idx, val = coo_to_csr(m_new, np.concatenate([brows, np.array(rows, np.int64)]),
                               np.concatenate([base.col_idx.astype(np.int64), np.array(cols, np.int64)]),
                               np.concatenate([base.values, np.array(vals)]))
    k = n_new - n
    return HostLP(m_new, n_new, ptr, idx, val, np.concatenate([base.c, c]), np.concatenate([base.AL, AL]),
                  np.concatenate([base.AU, AU]), np.concatenate([base.l, np.zeros(k)]),
                  np.concatenate([base.u, np.ones(k)])).ensure_transpose()


def _build(m, n, entries, c, AL, AU, l, u) -> HostLP:
    rows = np.array([r for r, _, _ in entries], np.int64)
    cols = np.array([j for _, j, _ in entries], np.int64)
    vals = np.array([a for _, _, a in entries], np.float64)
    ptr, idx, val = coo_to_csr(m, rows, cols, vals)
    return HostLP(m, n, ptr, idx, val, np.asarray(c, np.float64), np.asarray(AL, np.float64),
                  np.asarray(AU, np.float64), np.asarray(l, np.float64), np.asarray(u, np.float64)).ensure_transpose()


def _epigraph_pair(rng, t, e, r1, r2, entries, AL, AU, scale=None, mirror=None):
    """Rows r1, r2 reading  a t - a e >= 0  and  a t + a e >= 0  (a > 0), each
    row at random in its [0, inf) form or as its (-inf, 0] negation."""
    a = float(rng.choice([1.0, 2.0, 0.5])) if scale is None else scale
    for r, se in ((r1, -1.0), (r2, 1.0)):
        neg = bool(rng.random() < 0.5) if mirror is None else mirror
        k = -1.0 if neg else 1.0
        entries += [(r, t, k * a), (r, e, k * se * a)]
        AL[r], AU[r] = (-INF, 0.0) if neg else (0.0, INF)


def l1_split_lp(blocks: int, features: int, seed: int = 0, e_bounds: str = "free", decoy: str = "") -> HostLP:
    """L1 regression  min sum_i |r_i|,  r_i = b_i - a_i x, in the 3-row block
    layout the absolute-value reformulation's l1 split accepts: block i is the
    equality  a_i x + w_i e_i = b_i  and the pair  t_i >= |e_i|  (rows 3i,
    3i+1, 3i+2).  Feature columns x are free; every e_i is free
    (e_bounds="free"), in a finite box ("finite") or bounded below only
    ("lower").  Columns are shuffled so t and e come in both orders.
    `decoy` breaks one block: "coef" (an epigraph coefficient off by one
    ulp), "incidence" (t_0 also in block 1's equality), "shared" (block 1's
    pair reuses block 0's t)."""
    rng = np.random.default_rng(seed)
    n = features + 2 * blocks
    perm = rng.permutation(n)
    X = perm[:features]
    T = perm[features:features + blocks]
    E = perm[features + blocks:]
    m = 3 * blocks
    entries = []
    AL = np.zeros(m)
    AU = np.zeros(m)
    c = np.zeros(n)
    c[X] = np.round(rng.uniform(-0.1, 0.1, features), 3)
    c[T] = 1.0
    l = np.full(n, -INF)
    u = np.full(n, INF)
    l[T] = 0.0
    if e_bounds == "finite":
        l[E], u[E] = -50.0, 50.0
    elif e_bounds == "lower":
        l[E] = -50.0
    for i in range(blocks):
        k = int(rng.integers(1, min(features, 6) + 1))
        cols = rng.choice(X, size=k, replace=False)
        for j in cols:
            entries.append((3 * i, int(j), float(np.round(rng.uniform(-5, 5), 2) or 1.0)))
        entries.append((3 * i, int(E[i]), float(rng.choice([1.0, -1.0, 2.0]))))
        AL[3 * i] = AU[3 * i] = float(np.round(rng.uniform(-10, 10), 2))
        _epigraph_pair(rng, int(T[i]), int(E[i]), 3 * i + 1, 3 * i + 2, entries, AL, AU)
    if decoy == "coef":
        r, j, a = entries[-1]
        entries[-1] = (r, j, float(np.nextafter(a, 2 * a)))
    elif decoy == "incidence":
        entries.append((3, int(T[0]), 1.0))
    elif decoy == "shared":
        entries = [(r, int(T[0]) if (r in (4, 5) and j == int(T[1])) else j, a) for r, j, a in entries]
    return _build(m, n, entries, c, AL, AU, l, u)


def graph_l1_lp(blocks: int, features: int, seed: int = 0, group: int = 4, decoy: str = "") -> HostLP:
    """L1 model in the 4-row block layout of the graph variant: block i is the
    equality  a_i x + e_i = b_i,  the pair  t_i >= |e_i|  and  s - beta t_i >= 0
    for an auxiliary s shared by `group` consecutive blocks (zero cost,
    [0, inf)), so postsolve recovers s = max beta t.  `decoy`: "aux_cost"
    (one auxiliary has a cost), "extra_row" (block 0's fourth row has a
    third entry), "r3_sign" (a fourth row with the wrong sign)."""
    rng = np.random.default_rng(seed)
    aux = (blocks + group - 1) // group
    n = features + 2 * blocks + aux
    perm = rng.permutation(n)
    X = perm[:features]
    T = perm[features:features + blocks]
    E = perm[features + blocks:features + 2 * blocks]
    S = perm[features + 2 * blocks:]
    m = 4 * blocks
    entries = []
    AL = np.zeros(m)
    AU = np.zeros(m)
    c = np.zeros(n)
    c[X] = np.round(rng.uniform(-0.1, 0.1, features), 3)
    c[T] = np.round(rng.uniform(0.5, 2.0, blocks), 2)
    l = np.full(n, -INF)
    u = np.full(n, INF)
    l[T] = 0.0
    l[S] = 0.0
    for i in range(blocks):
        k = int(rng.integers(1, min(features, 6) + 1))
        for j in rng.choice(X, size=k, replace=False):
            entries.append((4 * i, int(j), float(np.round(rng.uniform(-5, 5), 2) or 1.0)))
        entries.append((4 * i, int(E[i]), float(rng.choice([1.0, -1.0, 3.0]))))
        AL[4 * i] = AU[4 * i] = float(np.round(rng.uniform(-10, 10), 2))
        _epigraph_pair(rng, int(T[i]), int(E[i]), 4 * i + 1, 4 * i + 2, entries, AL, AU, scale=1.0)
        beta = float(rng.choice([1.0, 0.5, 2.0, 1.5]))
        sgn = -1.0 if (decoy == "r3_sign" and i == blocks - 1) else 1.0
        entries += [(4 * i + 3, int(S[i // group]), sgn * 1.0), (4 * i + 3, int(T[i]), -beta)]
        AL[4 * i + 3], AU[4 * i + 3] = 0.0, INF
    if decoy == "aux_cost":
        c[S[0]] = 0.25
    elif decoy == "extra_row":
        entries.append((3, int(X[0]), 1.0))
    return _build(m, n, entries, c, AL, AU, l, u)


def outer_l1_lp(pairs: int, blocks: int, features: int = 6, seed: int = 0, share: bool = True,
                decoy: str = "") -> HostLP:
    """The outer-pair + linked-l1 layout: `pairs` 3-row groups forcing a free
    column f equal to a column b in [0, 10] (with `share`, every second pair
    reuses the previous b), then `blocks` 8-row blocks: an equality holding e
    and a few features (sometimes an outer free column), the pair q >= |e|
    on (e, q) with e's column before q's, the link alpha q - s = 0 and four
    rows x - s >= 0 on positive-cost columns x in [0, inf).  `decoy`:
    "dup_free" (two pairs share a free column), "role" (a block's q appears
    in another block's equality), "x_cost" (a zero-cost x)."""
    rng = np.random.default_rng(seed)
    entries = []
    AL, AU = [], []
    c, l, u = [], [], []

    def col(cost, lo, hi):
        c.append(cost)
        l.append(lo)
        u.append(hi)
        return len(c) - 1

    def row(ent, lo, hi):
        r = len(AL)
        entries.extend((r, j, a) for j, a in ent)
        AL.append(lo)
        AU.append(hi)

    bounds, frees = [], []
    for p in range(pairs):
        b = bounds[-1] if (share and p % 2 == 1) else col(float(np.round(rng.uniform(0.5, 3), 2)), 0.0, 10.0)
        f = col(float(np.round(rng.uniform(-1, 1), 2)), -INF, INF)
        if decoy == "dup_free" and p == 1:
            c.pop(); l.pop(); u.pop()
            f = frees[0]
        bounds.append(b)
        frees.append(f)
    feats = [col(float(np.round(rng.uniform(-0.1, 0.1), 3)), -INF, INF) for _ in range(features)]
    # Pair rows come after all columns exist so (b, f) is in column order.
    for b, f in zip(bounds, frees):
        assert b < f
        row([(b, 1.0), (f, -1.0)], 0.0, INF)
        row([(b, 1.0), (f, 1.0)], 0.0, INF)
        row([(b, -1.0), (f, 1.0)], 0.0, INF)
    qs = []
    for i in range(blocks):
        e = col(0.0, -INF, INF)
        q = col(float(np.round(rng.uniform(0.0, 1.0), 2)), 0.0, INF)
        s = col(0.0, 0.0, INF)
        xs = [col(0.0 if (decoy == "x_cost" and i == 0 and k == 0) else float(np.round(rng.uniform(0.1, 2), 2)),
                  0.0, INF) for k in range(4)]
        qs.append(q)
        dense = [(j, float(np.round(rng.uniform(-5, 5), 2) or 1.0))
                 for j in rng.choice(feats, size=min(3, features), replace=False)]
        if frees and rng.random() < 0.5:
            dense.append((int(rng.choice(frees)), 1.5))
        dense.append((e, float(rng.choice([1.0, -2.0]))))
        if decoy == "role" and i == 1:
            dense.append((qs[0], 1.0))
        rhs = float(np.round(rng.uniform(-10, 10), 2))
        row(dense, rhs, rhs)
        row([(e, -1.0), (q, 1.0)], 0.0, INF)
        row([(e, 1.0), (q, 1.0)], 0.0, INF)
        alpha = float(rng.choice([1.0, 0.5, 2.0]))
        row([(q, alpha), (s, -1.0)], 0.0, 0.0)
        for x in xs:
            row([(s, -1.0), (x, 1.0)], 0.0, INF)
    n = len(c)
    return _build(len(AL), n, entries, c, AL, AU, l, u)


def _pair_components(rng, P, size):
    """A random partition of P pairs into components of `size` pairs (the
    last may be smaller) and a spanning tree of each, plus one extra edge
    (a cycle) in every fourth component of three or more."""
    perm = rng.permutation(P)
    comps = [perm[i:i + size] for i in range(0, P, size)]
    edges = []
    for k, comp in enumerate(comps):
        for j in range(1, len(comp)):
            edges.append((int(comp[int(rng.integers(0, j))]), int(comp[j])))
        if len(comp) >= 3 and k % 4 == 0:
            edges.append((int(comp[0]), int(comp[-1])))
    owner = np.empty(P, np.int64)
    for k, comp in enumerate(comps):
        owner[comp] = k
    return comps, edges, owner


def _pair_row(rng, P, pairs, d, eq):
    """A row of pair terms  sum v_k (p_k - m_k)  with sides from the planted
    differences d: an equality or a one-sided row with slack."""
    v = np.round(rng.uniform(-4, 4, len(pairs)), 2)
    v[v == 0] = 1.0
    act = float(sum(vk * d[q] for vk, q in zip(v, pairs)))
    ent = [(int(q), float(vk)) for q, vk in zip(pairs, v)] + [(int(q) + P, float(-vk)) for q, vk in zip(pairs, v)]
    if eq:
        return ent, act, act
    return ent, act - float(rng.uniform(0.5, 2)), INF


def epigraph_pair_lp(components: int, size: int, tails: int = 2, rows: int = 0, seed: int = 0,
                     decoy: str = "") -> HostLP:
    """The variable-pair epigraph layout: P = components * size pairs (p_i =
    column i, m_i = column P + i, zero cost, [0, inf) or [0, u]), then `tails`
    positive-cost columns T.  Pair i's epigraph row  -a (p_i + m_i) + b T >= L
    shares (a, b, L, T) with its component; merge rows
    v (p_a - m_a) - v (p_b - m_b) = 0  join each component (a spanning tree,
    some with a cycle); `rows` (default P) further rows of 1-5 pair terms
    with sides from planted per-component differences.  Rows are shuffled.
    `decoy`: "epigraph_side" (one pair's L differs from its component's),
    "stray" (a row with a tail column in it)."""
    rng = np.random.default_rng(seed)
    P = components * size
    comps, edges, owner = _pair_components(rng, P, size)
    rows = P if rows == 0 else rows
    n = 2 * P + tails
    c = np.zeros(n)
    c[2 * P:] = np.round(rng.uniform(0.5, 2.0, tails), 2)
    l = np.zeros(n)
    u = np.full(n, INF)
    for k, comp in enumerate(comps):
        if k % 3 == 1:
            u[comp] = np.round(rng.uniform(20, 40, len(comp)), 1)
            u[comp + P] = np.round(rng.uniform(20, 40, len(comp)), 1)
    d = np.round(rng.uniform(-5, 5, len(comps)), 2)[owner]
    gdat = [(float(rng.choice([1.0, 2.0])), float(rng.choice([1.0, 0.5])), float(np.round(rng.uniform(-3, 0), 1)),
             2 * P + int(rng.integers(0, tails))) for _ in comps]
    body = []
    for i in range(P):
        a, b, L, t = gdat[owner[i]]
        if decoy == "epigraph_side" and i == int(comps[0][-1]) and len(comps[0]) > 1:
            L -= 1.0
        body.append(([(i, -a), (i + P, -a), (t, b)], L, INF))
    for x, y in edges:
        lo_, hi_ = min(x, y), max(x, y)
        v = float(rng.choice([1.0, -2.0, 0.5]))
        body.append(([(lo_, v), (hi_, -v), (lo_ + P, -v), (hi_ + P, v)], 0.0, 0.0))
    for r in range(rows):
        k = int(rng.integers(1, 6))
        pairs = rng.choice(P, size=k, replace=False)
        ent, lo_, hi_ = _pair_row(rng, P, pairs, d, eq=(r % 3 == 0))
        if decoy == "stray" and r == 0:
            ent.append((2 * P, 1.0))
            lo_, hi_ = -INF, INF
        body.append((ent, lo_, hi_))
    order = rng.permutation(len(body))
    entries, AL, AU = [], [], []
    for new, old in enumerate(order):
        ent, lo_, hi_ = body[old]
        entries += [(new, j, a) for j, a in ent]
        AL.append(lo_)
        AU.append(hi_)
    return _build(len(body), n, entries, c, AL, AU, l, u)


def antipodal_pair_lp(components: int, size: int, rows: int = 0, seed: int = 0, uniform_cost: bool = True,
                      decoy: str = "") -> HostLP:
    """The shifted-antipodal layout: P = components * size pairs, columns
    p_i = i and m_i = P + i only, costs c_p = c_m = rho (one value per
    component with `uniform_cost`, else per pair), lower bounds shared by a
    component (some nonzero, so the shift and the objective constant are
    exercised), finite or infinite uppers; merge rows joining each component
    and `rows` (default P) rows of 1-6 pair terms with sides from planted
    differences.  `decoy`: "shift" (a merge edge between components of
    different shifts), "cost" (one pair with c_p != c_m)."""
    rng = np.random.default_rng(seed)
    P = components * size
    comps, edges, owner = _pair_components(rng, P, size)
    rows = P if rows == 0 else rows
    n = 2 * P
    rho = np.round(rng.uniform(0.5, 3.0, len(comps)), 2)[owner] if uniform_cost else \
        np.round(rng.uniform(0.5, 3.0, P), 2)
    c = np.concatenate([rho, rho])
    lows = [(0.0, 0.0), (1.0, 1.0), (2.0, 0.5), (0.25, 0.75)]
    lp_, lm_ = np.zeros(P), np.zeros(P)
    for k, comp in enumerate(comps):
        lp_[comp], lm_[comp] = lows[k % len(lows)]
    l = np.concatenate([lp_, lm_])
    u = np.full(n, INF)
    for k, comp in enumerate(comps):
        if k % 3 == 2:
            u[comp] = l[comp] + 40.0
            u[comp + P] = l[comp + P] + 40.0
    if decoy == "cost":
        c[P] += 0.5
    d = np.round(rng.uniform(-5, 5, len(comps)), 2)[owner] + (lp_ - lm_)
    body = []
    if decoy == "shift":
        a, b = int(comps[0][0]), int(comps[2][0])   # shifts 0 and 1.5
        edges.append((a, b))
    for x, y in edges:
        lo_, hi_ = min(x, y), max(x, y)
        v = float(rng.choice([1.0, -2.0, 0.5]))
        body.append(([(lo_, v), (hi_, -v), (lo_ + P, -v), (hi_ + P, v)], 0.0, 0.0))
    for r in range(rows):
        k = int(rng.integers(1, 7))
        pairs = rng.choice(P, size=k, replace=False)
        body.append(_pair_row(rng, P, pairs, d, eq=(r % 3 == 0)))
    order = rng.permutation(len(body))
    entries, AL, AU = [], [], []
    for new, old in enumerate(order):
        ent, lo_, hi_ = body[old]
        entries += [(new, j, a) for j, a in ent]
        AL.append(lo_)
        AU.append(hi_)
    return _build(len(body), n, entries, c, AL, AU, l, u)


def workload(name: str, seed: int = 0) -> HostLP:
    """Named workloads: 'small' (2,000 x 5,000), 'scale' (2M x 5M + hubs), 'qap30',
    'random:MxN', 'slack:MxN' (random family with singleton columns on 30% of rows),
    'replicated:MxN*K' (K identical copies plus a coupling row), 'setcover:MxN' (unit set covering),
    'auxiliary:MxN' (random family plus projected-auxiliary blocks), 'qap:N', and the
    absolute-value layouts 'l1split:KxP' (K blocks, P features), 'graphl1:KxP' and
    'outerl1:PAIRSxBLOCKS', and the variable-pair layouts 'epigraph:CxS' / 'antipodal:CxS'
    (C components of S pairs)."""
    if name == "small":
        return random_lp(2000, 5000, seed)
    if name == "scale":
        return random_lp(2_000_000, 5_000_000, seed, hub_rows=2000)
    if name == "qap30":
        return qap_lp(30, seed)
    if name.startswith("random:"):
        m, n = (int(v) for v in name.split(":")[1].split("x"))
        return random_lp(m, n, seed)
    if name.startswith("slack:"):
        m, n = (int(v) for v in name.split(":")[1].split("x"))
        return random_lp(m, n, seed, slack_frac=0.3)
    if name.startswith("replicated:"):
        spec = name.split(":")[1]
        mn, k = spec.split("*")
        m, n = (int(v) for v in mn.split("x"))
        return replicated_lp(m, n, int(k), seed)
    if name.startswith("auxiliary:"):
        m, n = (int(v) for v in name.split(":")[1].split("x"))
        return auxiliary_lp(m, n, seed)
    if name.startswith("setcover:"):
        m, n = (int(v) for v in name.split(":")[1].split("x"))
        return setcover_lp(m, n, seed)
    if name.startswith("qap:"):
        return qap_lp(int(name.split(":")[1]), seed)
    if name.startswith("l1split:"):
        k, p = (int(v) for v in name.split(":")[1].split("x"))
        return l1_split_lp(k, p, seed)
    if name.startswith("graphl1:"):
        k, p = (int(v) for v in name.split(":")[1].split("x"))
        return graph_l1_lp(k, p, seed)
    if name.startswith("antipodal:"):
        k, size = (int(v) for v in name.split(":")[1].split("x"))
        return antipodal_pair_lp(k, size, seed=seed)
    if name.startswith("epigraph:"):
        k, size = (int(v) for v in name.split(":")[1].split("x"))
        return epigraph_pair_lp(k, size, seed=seed)
    if name.startswith("outerl1:"):
        pairs, blocks = (int(v) for v in name.split(":")[1].split("x"))
        return outer_l1_lp(pairs, blocks, seed=seed)
    raise ValueError(f"unknown workload {name!r}")


_MAGIC = b"GPPLP001"


def save_lp(path: str, lp: HostLP) -> None:
    """Binary LP file: magic, m, n, nnz, then A (CSR), c, l, u, AL, AU, obj_constant."""
    with open(path, "wb") as f:
        f.write(_MAGIC)
        f.write(struct.pack("<qqqd", lp.m, lp.n, lp.nnz, lp.obj_constant))
        for arr, dt in ((lp.row_ptr, np.int32), (lp.col_idx, np.int32), (lp.values, np.float64),
                        (lp.c, np.float64), (lp.l, np.float64), (lp.u, np.float64),
                        (lp.AL, np.float64), (lp.AU, np.float64)):
            f.write(np.ascontiguousarray(arr, dtype=dt).tobytes())


def load_lp(path: str) -> HostLP:
    with open(path, "rb") as f:
        if f.read(8) != _MAGIC:
            raise ValueError("not an LP file")
        m, n, nnz, obj = struct.unpack("<qqqd", f.read(32))
        rd = lambda k, dt: np.frombuffer(f.read(k * np.dtype(dt).itemsize), dtype=dt).copy()
        ptr, idx, val = rd(m + 1, np.int32), rd(nnz, np.int32), rd(nnz, np.float64)
        c, l, u, AL, AU = (rd(n, np.float64), rd(n, np.float64), rd(n, np.float64),
                           rd(m, np.float64), rd(m, np.float64))
    return HostLP(m, n, ptr, idx, val, c, AL, AU, l, u, obj).ensure_transpose()
