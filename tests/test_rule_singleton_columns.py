"""Singleton-column rule: the reference's known answers
(cpp/tests/test_rule_singleton_columns.cpp), on the oracle (CPU suite) and on
the CUDA engine through the C ABI (GPU suite)."""
import numpy as np
import pytest

from rule_cases import INF, Run, bits, make_lp

SCS, RDS = 2, 10   # SingletonColumnSubstitution, RowDualShift
RULE = ["singleton_columns"]
BACKENDS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


@pytest.mark.parametrize("backend", BACKENDS)
def test_eliminates_eq_singleton_column(backend):
    # test_eliminates_eq_singleton_column: x0 + x1 = 5, x1 fixed at 2.
    lp = make_lp(2, [[(0, 1.0), (1, 1.0)]], c=[4.0, 1.0], l=[0.0, 2.0], u=[10.0, 2.0], AL=[5.0], AU=[5.0])
    r = Run(backend, lp, RULE)
    assert (r.s.reduced_rows, r.s.reduced_cols) == (0, 1)
    assert r.col_map.tolist() == [1]
    assert abs(r.c[0] + 3.0) < 1e-12
    assert abs(r.s.obj_constant_delta - 20.0) < 1e-12
    t, idx, val = r.record(0)
    assert (t, idx) == (SCS, [0, 0, 1, 1])
    assert np.allclose(val, [1.0, 5.0, 0.0, 10.0, 4.0, 1.0, 1.0], atol=1e-12, rtol=0)
    assert len(r.tape_types) == 1


@pytest.mark.parametrize("backend", BACKENDS)
def test_eq_objective_updates_are_bitwise_deterministic(backend):
    # test_eq_objective_updates_are_bitwise_deterministic.
    lp = make_lp(3, [[(0, 3.0), (2, 0.1)], [(1, 7.0), (2, 0.2)]], c=[100000000.1, -99999999.9, 0.3],
                 l=[-INF, -INF, 0.0], u=[INF, INF, 0.0], AL=[5.0, 6.0], AU=[5.0, 6.0])
    expected = 0.3
    expected += -(100000000.1 * 0.1 / 3.0)
    expected += -(-99999999.9 * 0.2 / 7.0)
    for _ in range(4):
        r = Run(backend, lp, RULE)
        assert r.col_map.tolist() == [2]
        assert bits(r.c[0]) == bits(expected)


@pytest.mark.parametrize("backend", BACKENDS)
def test_dual_infer_marks_direct_unbounded(backend):
    lp = make_lp(2, [[(0, 1.0), (1, 1.0)]], c=[1.0, 0.0], l=[-INF, 0.0], u=[10.0, 1.0], AL=[-INF], AU=[5.0])
    r = Run(backend, lp, RULE)
    assert r.s.has_unbounded == 1


@pytest.mark.parametrize("backend", BACKENDS)
def test_dual_infer_records_row_dual_shift_then_eliminates(backend):
    # test_dual_infer_records_row_dual_shift_tape: the row becomes 1 <= x0 + x1
    # <= 1 with a RowDualShift record; the pipeline's next cleanup pass then
    # eliminates x0 from the new equality.
    lp = make_lp(2, [[(0, 1.0), (1, 1.0)]], c=[1.0, 0.0], l=[-INF, 0.0], u=[INF, 0.0], AL=[1.0], AU=[5.0])
    r = Run(backend, lp, RULE)
    t, idx, val = r.record(0)
    assert (t, idx) == (RDS, [0]) and val.tolist() == [0.0]
    t, idx, val = r.record(1)
    assert (t, idx) == (SCS, [0, 0, 1, 1])
    assert val[1] == 1.0


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("case", [
    # (objective, coefficient, lower, upper, lhs, rhs, expected side)
    (-1.0, 1.0, 10.0, 30.0, 5.0, 20.0, 20.0),    # c<0, a>0, implied free from above: upper side active
    (1.0, -1.0, 0.0, 10.0, -20.0, -5.0, -5.0),   # c>0, a<0, implied free from below: upper side active
    (1.0, 1.0, 0.0, 10.0, 5.0, 20.0, 5.0),       # c>0, a>0, implied free from below: lower side active
    (-1.0, -1.0, 10.0, 30.0, -20.0, -5.0, -20.0),  # c<0, a<0, implied free from above: lower side active
])
def test_dual_infer_tightens_one_sided_implied_free_row(backend, case):
    obj, a, lo, hi, lhs, rhs, side = case
    lp = make_lp(2, [[(0, a), (1, 1.0)]], c=[obj, 0.0], l=[lo, 0.0], u=[hi, 0.0], AL=[lhs], AU=[rhs])
    r = Run(backend, lp, RULE)
    t, idx, val = r.record(0)
    assert (t, idx) == (RDS, [0])
    t, idx, val = r.record(1)
    assert t == SCS and idx[:2] == [0, 0]
    assert abs(val[1] - side) < 1e-12


@pytest.mark.parametrize("backend", BACKENDS)
def test_unified_mixed_batch(backend):
    # test_unified_mixed_batch: batch 1 eliminates x0 and sets row 1's side,
    # batch 2 eliminates x1 from the inferred equality.
    lp = make_lp(3, [[(0, 1.0), (2, 1.0)], [(1, 1.0), (2, 1.0)]], c=[3.0, 2.0, 10.0], l=[-INF, -INF, 0.0],
                 u=[INF, INF, 2.0], AL=[5.0, 1.0], AU=[5.0, 7.0])
    r = Run(backend, lp, RULE)
    assert (r.s.reduced_rows, r.s.reduced_cols) == (0, 1)
    assert r.col_map.tolist() == [2] and r.c.tolist() == [5.0]
    assert r.s.obj_constant_delta == 17.0
    assert r.tape_types.tolist() == [SCS, RDS, SCS]
    assert r.tape_idx.tolist() == [0, 0, 1, 2, 1, 1, 1, 1, 2]
    assert r.tape_val.tolist() == [1.0, 5.0, -INF, INF, 3.0, 1.0, 1.0, 0.0, 1.0, 1.0, -INF, INF, 2.0, 1.0, 1.0]


@pytest.mark.parametrize("backend", BACKENDS)
def test_action_owner_prefers_free_then_smallest_column(backend):
    # test_action_owner_and_selective_commit: x0 is ineligible, x1 and x2
    # compete for the row and x1 (the smaller free pivot) wins.
    lp = make_lp(3, [[(0, 1.0), (1, 1.0), (2, 1.0)]], c=[-0.0, 3.0, 1.0], l=[0.0, -INF, -INF], u=[1.0, INF, INF],
                 AL=[5.0], AU=[5.0])
    r = Run(backend, lp, RULE)
    assert r.col_map.tolist() == [0, 2]
    assert bits(r.c).tolist() == bits([-3.0, -2.0]).tolist()
    assert r.s.obj_constant_delta == 15.0
    assert r.tape_types.tolist() == [SCS]
    assert r.tape_idx.tolist() == [1, 0, 2, 0, 2]


@pytest.mark.parametrize("backend", BACKENDS)
def test_unbounded_proposal_suppresses_batch(backend):
    lp = make_lp(4, [[(0, 1.0), (1, 1.0)], [(2, 1.0), (3, 1.0)]], c=[1.0, 0.0, -1.0, -0.0],
                 l=[-INF, 0.0, 10.0, 0.0], u=[10.0, 1.0, 30.0, 0.0], AL=[-INF, 5.0], AU=[5.0, 20.0])
    r = Run(backend, lp, RULE)
    assert r.s.has_unbounded == 1 and r.s.has_change == 0
    assert len(r.tape_types) == 0


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("m", [9, 1025])
def test_long_column_objective_order(backend, m):
    # test_long_column_objective_order: column m meets every eliminated row;
    # its cost update is summed in stored row order, bit for bit.
    n = m + 1
    rows, cost = [], [0.0] * n
    cost[m] = 0.3
    expected = cost[m]
    for row in range(m):
        pivot, coef = (7.0, 0.2) if row % 2 else (3.0, 0.1)
        rows.append([(row, pivot), (m, coef)])
        cost[row] = -99999999.9 if row % 2 else 100000000.1
        expected += -(cost[row] * coef / pivot)
    l, u = [-INF] * n, [INF] * n
    l[m] = u[m] = 0.0
    lp = make_lp(n, rows, c=cost, l=l, u=u, AL=[5.0] * m, AU=[5.0] * m)
    r = Run(backend, lp, RULE)
    assert r.s.has_infeasible == 0 and r.s.has_unbounded == 0
    assert r.col_map.tolist() == [m]
    assert bits(r.c[0]) == bits(expected)


@pytest.mark.parametrize("backend", BACKENDS)
def test_batched_substitution_tape(backend):
    # test_batched_singleton_column_substitution_tape_matches_cpu_oracle: rows
    # on both sides of the 1024 long-row threshold, mask holes, signed zero
    # coefficients and negative pivots.  The reference's masked-out columns
    # (j % 7 == 0) are fixed at zero here and removed by the fixed-variable rule
    # earlier in the same cleanup pass; the other non-pivot columns get [0, 1]
    # (the reference test holds them at [0, 0] with the fixed-variable rule
    # off), which changes no record.
    lengths = [1, 2, 1024, 1025, 2051, 3]
    rows, owner, rhs = [], [], []
    cost, lower, upper, keep, coeff_of = [], [], [], [], {}
    col = 0
    for row, length in enumerate(lengths):
        first = col
        pivot_col = first + (length - 1 if row % 2 else 0)
        pivot = -2.0 if row % 2 else 2.0
        owner.append(pivot_col)
        rhs.append(row + 1.0)
        entries = []
        for j in range(length):
            cj = first + j
            is_pivot = cj == pivot_col
            a = pivot if is_pivot else (-0.0 if j % 5 == 0 else (j % 3 - 1) * 0.25)
            entries.append((cj, a))
            coeff_of[cj] = a
            cost.append(row + 0.5 if is_pivot else 0.125)
            masked = not is_pivot and j % 7 == 0
            keep.append(not masked)
            lower.append(-INF if is_pivot else 0.0)
            upper.append(INF if is_pivot else (0.0 if masked else 1.0))
        rows.append(entries)
        col += length
    n = col
    lp = make_lp(n, rows, c=cost, l=lower, u=upper, AL=rhs, AU=rhs)
    r = Run(backend, lp, ["infeasible_and_fixed_variables", "singleton_columns"])
    types, idx, val = [], [], []
    for row, entries in enumerate(rows):
        pc = owner[row]
        support = [(cj, a) for cj, a in entries if cj != pc and keep[cj]]
        if not support:
            continue    # only the pivot left: a singleton row, not this rule's
        types.append(SCS)
        idx += [pc, row, len(support)] + [cj for cj, _ in support]
        val += [coeff_of[pc], rhs[row], -INF, INF, cost[pc], 1.0] + [a for _, a in support]
    assert r.tape_types.tolist() == types
    assert r.tape_idx.tolist() == idx
    assert bits(r.tape_val).tolist() == bits(val).tolist()
    # Surviving support columns: c_k - c_j a_k / a_j, bit for bit.
    got = dict(zip(r.col_map.tolist(), r.c.tolist()))
    for row, entries in enumerate(rows):
        pc = owner[row]
        if len(entries) == 1:
            continue
        for cj, a in entries:
            if cj == pc or not keep[cj]:
                continue
            e = 0.125
            e += -(cost[pc] * a / coeff_of[pc])
            assert bits(got[cj]) == bits(e), cj
