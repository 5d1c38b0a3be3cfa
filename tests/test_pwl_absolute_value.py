"""Absolute-value piecewise-linear reformulation (a Startup rule).

The known-answer cases are the reference's own rule tests
(cpp/tests/test_rule_piecewise_linear_reformulation_absolute_value.cpp:
L1SplitFixture :359-518, TwoGraphBlockFixture :520-575, the graph cases
:1080-1278, OuterFixture :119-293, OuterMappedDenseSortFixture :295-357),
restated as LPs.  They run through the whole pipeline with max_iters = 1, so
only Startup runs and the reduced model is the compacted form of the plan those
tests inspect; every case is also run on the reference library on the same GPU
(oracle/_ref/ref_driver) with the same settings and must agree in everything it
exports: reduced model, maps, tape, the primal-recovery checkpoints and the
recovery payload.  Generated models of each layout (lpgen.l1_split_lp,
graph_l1_lp, outer_l1_lp, with decoys) run the default pipeline against the
reference and against HiGHS (the postsolved optimum of the reduced model is
the original optimum).
"""
import numpy as np
import pytest

from gpp_b200 import capi, device, lpgen

import lpsolve
import test_reference_parity as trp

INF = np.inf
STARTUP = {"enable_structure_specific_rules": 1, "enable_piecewise_linear_reformulation_variable_pair": 0,
           "max_iters": 1}
PIPELINE = {"enable_structure_specific_rules": 1, "enable_piecewise_linear_reformulation_variable_pair": 0}
PATTERN = {"l1_split_3row": capi.ABS_L1_SPLIT, "graph_l1_substitution": capi.ABS_GRAPH_L1,
           "outer_pair_linked_l1": capi.ABS_OUTER_PAIR}


def host_lp(m, n, ptr, idx, val, c, l, u, AL, AU):
    return lpgen.HostLP(m, n, np.asarray(ptr, np.int32), np.asarray(idx, np.int32), np.asarray(val, np.float64),
                        np.asarray(c, np.float64), np.asarray(AL, np.float64), np.asarray(AU, np.float64),
                        np.asarray(l, np.float64), np.asarray(u, np.float64)).ensure_transpose()


# ---- the reference's fixtures --------------------------------------------------------------

def l1_fixture(variant="valid", lo=-INF, hi=INF):
    """L1SplitFixture: t=0, e=1, x=2;  e + 2x = 7,  t - e >= 0,  t + e >= 0."""
    c, l, u = [2.0, 0.5, 3.0], [0.0, lo, -INF], [INF, hi, INF]
    AL, AU = [7.0, 0.0, 0.0], [7.0, INF, INF]
    ptr, idx, val = [0, 2, 4, 6], [1, 2, 0, 1, 0, 1], [1.0, 2.0, 1.0, -1.0, 1.0, 1.0]
    m, n = 3, 3
    if variant == "t_in_equality":
        ptr, idx, val = [0, 3, 5, 7], [0, 1, 2, 0, 1, 0, 1], [0.25, 1.0, 2.0, 1.0, -1.0, 1.0, 1.0]
    elif variant == "duplicate_e":
        ptr, idx, val = [0, 3, 5, 7], [1, 1, 2, 0, 1, 0, 1], [0.5, 0.5, 2.0, 1.0, -1.0, 1.0, 1.0]
    elif variant == "near_coefficient":
        val = [1.0, 2.0, 1.0, -1.0 + 5.0e-13, 1.0, 1.0]
    elif variant == "tiny_rhs":
        AL = [7.0, 5.0e-13, 0.0]
    elif variant == "wrong_sign_infinity":
        AU = [7.0, -INF, INF]
    elif variant == "reverse_roles":
        # e=0, x=1, t=2.
        ptr, idx, val = [0, 2, 4, 6], [0, 1, 0, 2, 0, 2], [1.0, 2.0, -1.0, 1.0, 1.0, 1.0]
        c, l, u = [0.5, 3.0, 2.0], [lo, -INF, 0.0], [hi, INF, INF]
    elif variant == "shared_roles":
        m, n = 6, 4
        ptr, idx = [0, 2, 4, 6, 8, 10, 12], [1, 2, 0, 1, 0, 1, 1, 3, 0, 1, 0, 1]
        val = [1.0, 2.0, 1.0, -1.0, 1.0, 1.0, 1.0, 3.0, 1.0, -1.0, 1.0, 1.0]
        c, l, u = [2.0, 0.5, 3.0, 4.0], [0.0, lo, -INF, -INF], [INF, hi, INF, INF]
        AL, AU = [7.0, 0.0, 0.0, 9.0, 0.0, 0.0], [7.0, INF, INF, 9.0, INF, INF]
    elif variant == "second_t_bound":
        m, n = 6, 6
        ptr, idx = [0, 2, 4, 6, 8, 10, 12], [1, 4, 0, 1, 0, 1, 3, 5, 2, 3, 2, 3]
        val = [1.0, 2.0, 1.0, -1.0, 1.0, 1.0, 1.0, 3.0, 1.0, -1.0, 1.0, 1.0]
        c = [2.0, 0.5, 4.0, 0.75, 3.0, 5.0]
        l, u = [0.0, lo, 5.0e-13, lo, -INF, -INF], [INF, hi, INF, hi, INF, INF]
        AL, AU = [7.0, 0.0, 0.0, 9.0, 0.0, 0.0], [7.0, INF, INF, 9.0, INF, INF]
    elif variant == "trailing_empty_row":
        m, ptr, AL, AU = 4, ptr + [ptr[-1]], AL + [0.0], AU + [INF]
    return host_lp(m, n, ptr, idx, val, c, l, u, AL, AU)


def graph_fixture():
    """The four-row graph block (:1080-1098): t=0, e=1, s=2."""
    return host_lp(4, 3, [0, 1, 3, 5, 7], [1, 0, 1, 0, 1, 0, 2], [3.0, 1.0, -1.0, 1.0, 1.0, -2.0, 1.0],
                   [0.5, 2.0, 0.0], [0.0, -INF, 0.0], [INF, INF, INF], [7.0, 0.0, 0.0, 0.0], [7.0, INF, INF, INF])


def shared_aux_fixture(invalid=0):
    """Two blocks sharing the auxiliary s=4 (:1177-1278); invalid 1 gives s a
    cost, 2 an upper bound."""
    ptr = [0, 1, 3, 5, 7, 8, 10, 12, 14]
    idx = [1, 0, 1, 0, 1, 0, 4, 3, 2, 3, 2, 3, 2, 4]
    val = [3.0, 1.0, -1.0, 1.0, 1.0, -2.0, 1.0, 4.0, 1.0, -1.0, 1.0, 1.0, -3.0, 1.0]
    c = [0.5, 2.0, 0.75, 1.25, 1.0 if invalid == 1 else 0.0]
    u = [INF, INF, INF, INF, 10.0 if invalid == 2 else INF]
    return host_lp(8, 5, ptr, idx, val, c, [0.0, -INF, 0.0, -INF, 0.0], u,
                   [7.0, 0.0, 0.0, 0.0, 11.0, 0.0, 0.0, 0.0], [7.0, INF, INF, INF, 11.0, INF, INF, INF])


def two_graph_block_fixture():
    """Block 0 valid, block 1's e in a finite box: the whole match fails."""
    ptr = [0, 1, 3, 5, 7, 8, 10, 12, 14]
    idx = [1, 0, 1, 0, 1, 0, 2, 4, 3, 4, 3, 4, 3, 5]
    val = [3.0, 1.0, -1.0, 1.0, 1.0, -2.0, 1.0, 4.0, 1.0, -1.0, 1.0, 1.0, -3.0, 1.0]
    return host_lp(8, 6, ptr, idx, val, [0.5, 2.0, 0.0, 0.75, 1.25, 0.0], [0.0, -INF, 0.0, 0.0, -5.0, 0.0],
                   [INF, INF, INF, INF, 5.0, INF], [7.0, 0.0, 0.0, 0.0, 11.0, 0.0, 0.0, 0.0],
                   [7.0, INF, INF, INF, 11.0, INF, INF, INF])


def outer_fixture(variant="shared_bound"):
    """OuterFixture: a=0, b=1, c=2 (b = a and c = a), e=3, q=4, s=5, x1..x4=6..9."""
    rows = [[(0, 1.0), (1, -1.0)], [(0, 1.0), (1, 1.0)], [(0, -1.0), (1, 1.0)],
            [(0, 1.0), (2, -1.0)], [(0, 1.0), (2, 1.0)], [(0, -1.0), (2, 1.0)],
            [(3, 1.0)], [(3, -1.0), (4, 1.0)], [(3, 1.0), (4, 1.0)], [(4, 1.0), (5, -1.0)],
            [(5, -1.0), (6, 1.0)], [(5, -1.0), (7, 1.0)], [(5, -1.0), (8, 1.0)], [(5, -1.0), (9, 1.0)]]
    c = [1.0, 2.0, 3.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0]
    l = [0.0, -INF, -INF, -INF, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0]
    u = [10.0] + [INF] * 9
    AU = [INF] * 6 + [0.0, INF, INF, 0.0, INF, INF, INF, INF]
    n = 10

    def second_block():
        nonlocal n
        rows.extend([[(10, 1.0)], [(10, -1.0), (11, 1.0)], [(10, 1.0), (11, 1.0)], [(11, 1.0), (12, -1.0)],
                     [(12, -1.0), (6, 1.0)], [(12, -1.0), (7, 1.0)], [(12, -1.0), (8, 1.0)], [(12, -1.0), (9, 1.0)]])
        c.extend([0.0, 0.0, 0.0])
        l.extend([-INF, 0.0, 0.0])
        u.extend([INF, INF, INF])
        AU.extend([0.0, INF, INF, 0.0, INF, INF, INF, INF])
        n = 13

    if variant == "two_blocks":
        second_block()
    elif variant == "duplicate_free":
        for r in (3, 4, 5):
            rows[r] = [(0, rows[r][0][1]), (1, rows[r][1][1])]
    elif variant == "bound_free_overlap":
        for r in (3, 4, 5):
            rows[r] = [(1, rows[r][0][1]), (2, rows[r][1][1])]
    elif variant == "outer_block_role":
        # The block's e is the outer free column b.
        rows[6], rows[7], rows[8] = [(1, 1.0)], [(1, -1.0), (4, 1.0)], [(1, 1.0), (4, 1.0)]
    elif variant == "dense_own_q":
        rows[6] = [(3, 1.0), (4, 2.0)]
    elif variant == "dense_own_s":
        rows[6] = [(3, 1.0), (5, 2.0)]
    elif variant == "dense_duplicate_e":
        rows[6] = [(3, 1.0), (3, 2.0)]
    elif variant == "dense_mapped_duplicate":
        rows[6] = [(1, 2.0), (2, 3.0), (3, 1.0)]
    elif variant in ("dense_cross_q", "dense_cross_e", "dense_cross_s"):
        second_block()
        rows[6] = [(3, 1.0), ({"dense_cross_e": 10, "dense_cross_q": 11, "dense_cross_s": 12}[variant], 2.0)]
    m = len(rows)
    ptr = np.cumsum([0] + [len(r) for r in rows])
    idx = [j for r in rows for j, _ in r]
    val = [a for r in rows for _, a in r]
    return host_lp(m, n, ptr, idx, val, c, l, u, [0.0] * m, AU)


def outer_sort_fixture():
    """OuterMappedDenseSortFixture: bound=0, free=9, e=1, q=2, s=3, x=4..7."""
    ptr = [0, 2, 4, 6, 9, 11, 13, 15, 17, 19, 21, 23]
    idx = [0, 9, 0, 9, 0, 9, 1, 8, 9, 1, 2, 1, 2, 2, 3, 3, 4, 3, 5, 3, 6, 3, 7]
    val = [1.0, -1.0, 1.0, 1.0, -1.0, 1.0, 1.0, 5.0, 2.0, -1.0, 1.0, 1.0, 1.0, 1.0, -1.0, -1.0, 1.0, -1.0, 1.0,
           -1.0, 1.0, -1.0, 1.0]
    return host_lp(11, 10, ptr, idx, val, [1.0, 0.5, 0.25, 0.75, 1.0, 1.0, 1.0, 1.0, 3.0, 2.0],
                   [0.0, -INF, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -INF, -INF], [10.0] + [INF] * 9,
                   [0.0, 0.0, 0.0, 7.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0],
                   [INF, INF, INF, 7.0, INF, INF, 0.0, INF, INF, INF, INF])


# ---- reference comparison of the recovery data --------------------------------------------------

def check_recoveries(got):
    """Checkpoints and absolute-value payloads equal the reference's."""
    ref = got.ref
    rk = trp_file(ref, "ckpt_kind", np.int32)
    rp = trp_file(ref, "ckpt_payload", np.int32)
    rq = trp_file(ref, "ckpt_position", np.int64)
    assert got.checkpoints == list(zip(rk.tolist(), rp.tolist(), rq.tolist()))
    assert len(got.absolute_value) == int(ref["meta"]["absolute_value_steps"])
    for k, a in enumerate(got.absolute_value):
        assert a["pattern"] == PATTERN[ref["meta"][f"abs{k}_pattern"]]
        for key, dt in (("split_t", np.int32), ("split_e", np.int32), ("split_rho", np.float64),
                        ("pair_bound", np.int32), ("pair_free", np.int32), ("link_slack", np.int32),
                        ("link_t", np.int32), ("link_factor", np.float64), ("max_slack", np.int32),
                        ("max_start", np.int32), ("max_t", np.int32), ("max_factor", np.float64)):
            want = trp_file(ref, f"abs{k}_{key}", dt)
            have = a[key] if not (key == "max_start" and len(a["max_slack"]) == 0) else np.zeros(1, np.int32)
            assert np.array_equal(have, want), key


def trp_file(ref, name, dt):
    import os
    return np.fromfile(os.path.join(ref["dir"], name), dtype=dt)


def presolve_vs_reference(lp, extra, postsolve=False):
    """Startup-only settings (max_iters in `extra`) also turn every other rule
    off, so the reduced model is exactly the reformulation's rewrite."""
    rules = [] if extra.get("max_iters") == 1 else trp.ALL
    got = trp.check_against_reference(lp, rules, extra, oracle=False, postsolve=postsolve)
    check_recoveries(got)
    return got


# ---- tests ------------------------------------------------------------------------------------

pytestmark = pytest.mark.gpu


def test_exports_and_restore_symbols():
    lib = capi.load()
    for name in ("gpp_recovery_checkpoints", "gpp_absolute_value_sizes", "gpp_export_absolute_value",
                 "gpp_restore_absolute_value"):
        assert hasattr(lib, name)


@trp.needs_reference
@pytest.mark.parametrize("lo,hi,mode,rows_kept", [
    (-2.0, 2.0, 0, 2), (-INF, INF, 0, 1), (-INF, 5.0, 0, 2), (-1.0e9, 1.0e9, 2, 1), (-2.0, 2.0, 1, 3)])
def test_l1_split_known_answers(lo, hi, mode, rows_kept):
    """Finite residual bounds keep  l_e <= p - q <= u_e  (preserve mode), a
    free residual goes 3 rows to 1, the legacy mode treats a wide box as
    free, and the strict mode rejects a bounded residual."""
    extra = {**STARTUP, "piecewise_linear_reformulation_absolute_value_residual_bound_mode": mode}
    got = presolve_vs_reference(l1_fixture("valid", lo, hi), extra)
    s = got.summary
    assert s.reduced_rows == rows_kept
    if rows_kept == 3:
        assert got.checkpoints == [] and got.absolute_value == []
        return
    assert np.array_equal(got.c, [2.5, 1.5, 3.0])
    assert np.array_equal(got.A_ptr[:2], [0, 3]) and np.array_equal(got.A_idx[:3], [0, 1, 2])
    assert np.array_equal(got.A_val[:3], [1.0, -1.0, 2.0])
    if rows_kept == 2:
        assert np.array_equal(got.A_idx[3:], [0, 1]) and np.array_equal(got.A_val[3:], [1.0, -1.0])
        assert got.AL[1] == lo and got.AU[1] == hi
    (a,) = got.absolute_value
    assert a["pattern"] == capi.ABS_L1_SPLIT
    assert a["split_t"].tolist() == [0] and a["split_e"].tolist() == [1] and a["split_rho"].tolist() == [1.0]
    assert got.checkpoints == [(0, 0, 0)]


@trp.needs_reference
@pytest.mark.parametrize("variant", ["t_in_equality", "duplicate_e", "near_coefficient", "tiny_rhs",
                                     "wrong_sign_infinity", "shared_roles", "second_t_bound",
                                     "trailing_empty_row"])
def test_l1_split_fails_closed(variant):
    lp = l1_fixture(variant, -INF, INF)
    got = presolve_vs_reference(lp, STARTUP)
    assert (got.summary.reduced_rows, got.summary.reduced_cols) == (lp.m, lp.n)
    assert got.checkpoints == []


@trp.needs_reference
def test_l1_split_reverse_role_order_is_sorted():
    got = presolve_vs_reference(l1_fixture("reverse_roles", -2.0, 2.0), STARTUP)
    for i in range(got.summary.reduced_rows):
        row = got.A_idx[got.A_ptr[i]:got.A_ptr[i + 1]]
        assert np.all(np.diff(row) > 0)
    assert got.absolute_value[0]["split_t"].tolist() == [2]


@trp.needs_reference
def test_graph_known_answer_and_restore():
    import torch
    got = presolve_vs_reference(graph_fixture(), STARTUP)
    assert (got.summary.reduced_rows, got.summary.reduced_cols) == (1, 2)
    assert got.A_idx.tolist() == [0, 1] and got.A_val.tolist() == [3.0, -3.0]
    assert got.c.tolist() == [2.5, -1.5]
    (a,) = got.absolute_value
    assert a["pattern"] == capi.ABS_GRAPH_L1 and a["max_slack"].tolist() == [2]
    # The reference test's restore: (4, 1, 0) -> (5, 3, 10).
    x = torch.tensor([4.0, 1.0, 0.0], dtype=torch.float64, device="cuda")
    low = torch.tensor([0.0, -INF, 0.0], dtype=torch.float64, device="cuda")
    device.restore_absolute_value(x, got.absolute_value, low)
    assert x.cpu().tolist() == [5.0, 3.0, 10.0]


@trp.needs_reference
@pytest.mark.parametrize("invalid", [0, 1, 2])
def test_graph_shared_auxiliary(invalid):
    import torch
    lp = shared_aux_fixture(invalid)
    got = presolve_vs_reference(lp, STARTUP)
    if invalid:
        assert (got.summary.reduced_rows, got.summary.reduced_cols) == (lp.m, lp.n)
        return
    assert (got.summary.reduced_rows, got.summary.reduced_cols) == (2, 4)
    assert got.A_idx.tolist() == [0, 1, 2, 3] and got.A_val.tolist() == [3.0, -3.0, 4.0, -4.0]
    assert got.c.tolist() == [2.5, -1.5, 2.0, -0.5]
    (a,) = got.absolute_value
    assert a["max_slack"].tolist() == [4] and a["max_t"].tolist() == [0, 2]
    assert a["max_factor"].tolist() == [2.0, 3.0]
    x = torch.tensor([4.0, 1.0, 2.0, 1.0, 0.0], dtype=torch.float64, device="cuda")
    low = torch.tensor([0.0, -INF, 0.0, -INF, 0.0], dtype=torch.float64, device="cuda")
    device.restore_absolute_value(x, got.absolute_value, low)
    assert x.cpu().tolist() == [5.0, 3.0, 3.0, 1.0, 10.0]


@trp.needs_reference
def test_graph_mixed_validity_fails_closed():
    lp = two_graph_block_fixture()
    got = presolve_vs_reference(lp, STARTUP)
    assert (got.summary.reduced_rows, got.summary.reduced_cols) == (lp.m, lp.n)


@trp.needs_reference
def test_outer_shared_bound_known_answer():
    import torch
    got = presolve_vs_reference(outer_fixture("shared_bound"), STARTUP)
    (a,) = got.absolute_value
    assert a["pattern"] == capi.ABS_OUTER_PAIR
    assert a["pair_bound"].tolist() == [0, 0] and a["pair_free"].tolist() == [1, 2]
    assert got.c[0] == 6.0   # 1 + 2 + 3, in pair order
    # Kept: rows 6 and 10-13, columns all but b, c and s.
    assert got.row_map.tolist() == [6, 10, 11, 12, 13]
    assert got.col_map.tolist() == [0, 3, 4, 6, 7, 8, 9]
    assert got.A_ptr.tolist() == [0, 2, 5, 8, 11, 14]
    # The reference test's primal restore: a = 2.25 gives b = c = 2.25.
    x = torch.zeros(10, dtype=torch.float64, device="cuda")
    x[0] = 2.25
    device.restore_absolute_value(x, got.absolute_value)
    assert x[1].item() == 2.25 and x[2].item() == 2.25


@trp.needs_reference
def test_outer_mapped_dense_row_is_sorted():
    got = presolve_vs_reference(outer_sort_fixture(), STARTUP)
    (a,) = got.absolute_value
    assert a["split_t"].tolist() == [2] and a["split_e"].tolist() == [1]
    assert a["pair_bound"].tolist() == [0] and a["pair_free"].tolist() == [9]
    assert got.row_map.tolist() == [3, 7, 8, 9, 10]
    # The dense row [e=1, z=8, free=9] becomes [0: 2, 1: -1, 2: 1, 8: 5].
    assert got.A_idx[:4].tolist() == [0, 1, 2, 7] and got.A_val[:4].tolist() == [2.0, -1.0, 1.0, 5.0]


@trp.needs_reference
@pytest.mark.parametrize("variant", ["two_blocks", "duplicate_free", "bound_free_overlap", "outer_block_role",
                                     "dense_own_q",
                                     "dense_own_s", "dense_duplicate_e", "dense_mapped_duplicate",
                                     "dense_cross_q", "dense_cross_e", "dense_cross_s"])
def test_outer_variants(variant):
    lp = outer_fixture(variant)
    got = presolve_vs_reference(lp, STARTUP)
    if variant == "two_blocks":
        (a,) = got.absolute_value
        assert len(a["split_t"]) == 2 and len(a["link_slack"]) == 2
    else:
        assert got.checkpoints == []
        assert (got.summary.reduced_rows, got.summary.reduced_cols) == (lp.m, lp.n)


@trp.needs_reference
@pytest.mark.parametrize("maker,kw", [
    (lpgen.l1_split_lp, dict(blocks=400, features=30)),
    (lpgen.l1_split_lp, dict(blocks=400, features=30, e_bounds="finite")),
    (lpgen.l1_split_lp, dict(blocks=400, features=30, e_bounds="lower")),
    (lpgen.l1_split_lp, dict(blocks=300, features=20, decoy="coef")),
    (lpgen.l1_split_lp, dict(blocks=300, features=20, decoy="incidence")),
    (lpgen.l1_split_lp, dict(blocks=300, features=20, decoy="shared")),
    (lpgen.graph_l1_lp, dict(blocks=400, features=30)),
    (lpgen.graph_l1_lp, dict(blocks=400, features=30, group=1)),
    (lpgen.graph_l1_lp, dict(blocks=300, features=20, decoy="aux_cost")),
    (lpgen.graph_l1_lp, dict(blocks=300, features=20, decoy="extra_row")),
    (lpgen.graph_l1_lp, dict(blocks=300, features=20, decoy="r3_sign")),
    (lpgen.outer_l1_lp, dict(pairs=40, blocks=200)),
    (lpgen.outer_l1_lp, dict(pairs=40, blocks=200, share=False)),
    (lpgen.outer_l1_lp, dict(pairs=20, blocks=100, decoy="dup_free")),
    (lpgen.outer_l1_lp, dict(pairs=20, blocks=100, decoy="role")),
    (lpgen.outer_l1_lp, dict(pairs=20, blocks=100, decoy="x_cost")),
])
@pytest.mark.parametrize("seed", [0, 1])
def test_generated_layouts_match_reference(maker, kw, seed):
    """Default pipeline (all rules, folding off) on each layout: the same
    reduced model, tape, checkpoints and recovery payloads as the reference,
    and the same postsolved point."""
    lp = maker(**kw, seed=seed)
    got = presolve_vs_reference(lp, PIPELINE, postsolve=True)
    fires = not kw.get("decoy")
    assert (len(got.checkpoints) == 1) == fires


@trp.needs_reference
def test_reference_variable_pair_detector_rejects_these_layouts():
    """With the reference's defaults (variable-pair reformulation on) its
    output on these models equals its output with that rule off, so the
    engine matches the reference's default settings here too."""
    for lp in (lpgen.l1_split_lp(400, 30, seed=0), lpgen.graph_l1_lp(400, 30, seed=0),
               lpgen.outer_l1_lp(40, 200, seed=0)):
        on = trp.run_reference(lp, trp.ALL, ["enable_structure_specific_rules=1"])
        off = trp.run_reference(lp, trp.ALL, ["enable_structure_specific_rules=1",
                                              "enable_piecewise_linear_reformulation_variable_pair=0"])
        for k in ("row_map", "col_map", "A_idx", "tape_types"):
            assert np.array_equal(on[k], off[k]), k


@pytest.mark.parametrize("maker,kw", [
    (lpgen.l1_split_lp, dict(blocks=200, features=15)),
    (lpgen.l1_split_lp, dict(blocks=200, features=15, e_bounds="finite")),
    (lpgen.graph_l1_lp, dict(blocks=200, features=15)),
    (lpgen.outer_l1_lp, dict(pairs=20, blocks=100)),
])
def test_postsolved_optimum_is_the_original_one(maker, kw):
    """HiGHS on the original model and on the reduced one: the postsolved
    reduced optimum is feasible for the original model and has its optimal
    objective."""
    import torch
    lp = maker(**kw, seed=3)
    params = capi.params_with_rules(trp.ALL, enable_folding=0, **PIPELINE)
    dlp = device.DeviceLp(lp)
    s = device.preprocess(dlp, params)
    try:
        got = device.Result(s)
        assert len(got.checkpoints) == 1
        res0, _, _ = lpsolve.solve(lp.m, lp.n, lp.row_ptr, lp.col_idx, lp.values, lp.c, lp.AL, lp.AU, lp.l, lp.u)
        rr, yr, zr = lpsolve.solve(s.reduced_rows, s.reduced_cols, got.A_ptr, got.A_idx, got.A_val, got.c, got.AL,
                                   got.AU, got.l, got.u)
        assert res0.status == 0 and rr.status == 0
        x, _, _ = device.postprocess(torch.from_numpy(rr.x).cuda(), torch.from_numpy(yr).cuda(),
                                     torch.from_numpy(zr).cuda(), s, dlp)
        x = np.asarray(x)
        assert abs(lp.c @ x + lp.obj_constant - res0.fun) <= 1e-7 * max(1.0, abs(res0.fun))
        assert lpsolve.primal_violation(lp, x) <= 1e-7
    finally:
        device.free_summary(s)
