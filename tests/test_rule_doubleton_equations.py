"""Doubleton-equation rule (batch mode): the reference's known answers
(cpp/tests/test_rule_doubleton_equations.cpp), on the oracle (CPU suite) and
on the CUDA engine through the C ABI (GPU suite).  Small batches are allowed
(min_selected_per_batch = 1, ratio 0), as in those tests."""
import numpy as np
import pytest

from rule_cases import INF, Run, make_lp

DOUBLETON = 13
RULE = ["doubleton_equations"]
SMALL_BATCH = dict(doubleton_equations_min_selected_per_batch=1, doubleton_equations_min_selected_ratio=0.0)
BACKENDS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


@pytest.mark.parametrize("backend", BACKENDS)
def test_batch_records_exact_doubleton_tape(backend):
    # test_batch_records_exact_doubleton_tape and, through the batch path, the
    # outcome of test_eliminates_doubleton_equation_row: x0 + 2 x1 = 4.
    lp = make_lp(2, [[(0, 1.0), (1, 2.0)]], c=[3.0, 5.0], l=[0.0, -INF], u=[10.0, INF], AL=[4.0], AU=[4.0])
    r = Run(backend, lp, RULE, **SMALL_BATCH)
    assert (r.s.reduced_rows, r.s.reduced_cols) == (0, 1)
    assert r.col_map.tolist() == [1]
    assert abs(r.c[0] - (-1.0)) < 1e-12
    assert abs(r.s.obj_constant_delta - 12.0) < 1e-12
    assert (r.l[0], r.u[0]) == (-3.0, 2.0)
    assert r.tape_types.tolist() == [DOUBLETON]
    assert r.tape_idx.tolist() == [0, 1, 0, 0]
    expected = [1.0, 2.0, 4.0, 0.0, 10.0, -INF, INF, -3.0, 2.0, 3.0, 0.0, 0.0]
    for got, want in zip(r.tape_val.tolist(), expected):
        if np.isinf(want):
            assert got == want
        else:
            assert abs(got - want) < 1e-12


def fill_cap_lp():
    # Row 0 is x0 + x1 = 0; x0 has 12 more rows and x1 has 13, so x0 is
    # eliminated and its fill proxy is 11.
    rows = [[(0, 1.0), (1, 1.0)]] + [[(0, 1.0)] for _ in range(12)] + [[(1, 1.0)] for _ in range(13)]
    m = len(rows)
    AL = [-INF] * m
    AU = [INF] * m
    AL[0] = AU[0] = 0.0
    return make_lp(2, rows, c=[0.0, 0.0], l=[-INF, -INF], u=[INF, INF], AL=AL, AU=AU)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("cap,changed", [(10, False), (96, True)])
def test_fill_cap(backend, cap, changed):
    # test_default_fill_cap_accepts_more_than_ten.
    r = Run(backend, fill_cap_lp(), RULE, doubleton_equations_max_fill_in_proxy=cap, **SMALL_BATCH)
    assert bool(r.s.has_change) == changed
    if changed:
        assert 0 not in r.row_map.tolist() and r.col_map.tolist() == [1]


@pytest.mark.parametrize("backend", BACKENDS)
def test_one_batch_leaves_conflicting_equation_for_later(backend):
    # x0 + x1 = 1 and x1 + x2 = 2 share x1: only the first is substituted.
    lp = make_lp(3, [[(0, 1.0), (1, 1.0)], [(1, 1.0), (2, 1.0)]], c=[3.0, 5.0, 7.0], l=[-INF] * 3, u=[INF] * 3,
                 AL=[1.0, 2.0], AU=[1.0, 2.0])
    r = Run(backend, lp, RULE, **SMALL_BATCH)
    assert r.row_map.tolist() == [1] and r.col_map.tolist() == [1, 2]
    assert abs(r.c[0] - 2.0) < 1e-12 and abs(r.c[1] - 7.0) < 1e-12
    assert abs(r.s.obj_constant_delta - 3.0) < 1e-12
    assert r.tape_types.tolist() == [DOUBLETON]


@pytest.mark.parametrize("backend", BACKENDS)
def test_batch_below_minimum_is_skipped(backend):
    # Defaults: fewer than 256 selected rows leave the model unchanged.
    lp = make_lp(2, [[(0, 1.0), (1, 2.0)]], c=[3.0, 5.0], l=[0.0, -INF], u=[10.0, INF], AL=[4.0], AU=[4.0])
    r = Run(backend, lp, RULE)
    assert r.s.has_change == 0 and len(r.tape_types) == 0


@pytest.mark.parametrize("backend", BACKENDS)
def test_keep_column_fixed_when_bounds_close(backend):
    # x0 - x1 = 0: both columns have two rows, so x1 is eliminated and x0
    # kept.  x0 in [2, 2 + 1e-10] is closed within bound_tol, so x0 is fixed
    # at the midpoint instead, the row stays (a singleton row in x1 after the
    # shift) and there is no DoubletonEquation record.
    lp = make_lp(2, [[(0, 1.0), (1, -1.0)], [(0, 1.0), (1, 1.0)]], c=[1.0, 2.0], l=[2.0, -INF],
                 u=[2.0 + 1e-10, INF], AL=[0.0, -INF], AU=[0.0, 10.0])
    r = Run(backend, lp, RULE, **SMALL_BATCH)
    assert r.s.has_change == 1
    assert len(r.tape_types) == 0
    assert r.fixed_idx.tolist() == [0]
    assert r.row_map.tolist() == [0, 1] and r.col_map.tolist() == [1]
    assert abs(r.AU[0] - (0.0 - 1.0 * (2.0 + 0.5e-10))) < 1e-15


@pytest.mark.parametrize("backend", BACKENDS)
def test_eliminates_doubleton_equation_row_single_row_mode(backend):
    # test_eliminates_doubleton_equation_row: doubleton_equations_scan = 0.
    lp = make_lp(2, [[(0, 1.0), (1, 2.0)]], c=[3.0, 5.0], l=[0.0, -INF], u=[10.0, INF], AL=[4.0], AU=[4.0])
    r = Run(backend, lp, RULE, doubleton_equations_scan=0, doubleton_equations_max_fill_in_proxy=10)
    assert r.row_map.tolist() == [] and r.col_map.tolist() == [1]
    assert abs(r.c[0] - (-1.0)) < 1e-12
    assert abs(r.s.obj_constant_delta - 12.0) < 1e-12
    assert r.tape_types.tolist() == [DOUBLETON]


@pytest.mark.parametrize("backend", BACKENDS)
def test_single_row_mode_substitutes_one_row_per_call(backend):
    # Two independent doubletons: one substitution per rule call, the smallest
    # row first; the scheduler's next aggregation round takes the other only
    # after nnz progress, which this tiny LP never makes.
    lp = make_lp(4, [[(0, 1.0), (1, 1.0)], [(2, 1.0), (3, 2.0)]], c=[1.0, 2.0, 3.0, 4.0], l=[-INF] * 4,
                 u=[INF] * 4, AL=[1.0, 2.0], AU=[1.0, 2.0])
    r = Run(backend, lp, RULE, doubleton_equations_scan=0)
    assert r.tape_types.tolist() == [DOUBLETON]
    assert r.tape_idx.tolist()[2] == 0
