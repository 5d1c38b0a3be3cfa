"""Parity with the reference library at benchmark size, on the GPU.

The benchmark LP (the random family at m = 2,000,000, n = 5,000,000 plus
2,000 hub rows, 29.8M nnz) and the QAP N = 30 Adams-Johnson LP (1,674,960
rows, 810,900 columns) are presolved by the engine and by the reference
library with the benchmark's parameters: every rule of the plain path,
folding on, the structure-specific startup rules at their defaults.  The
removed sets, maps, sparsity patterns, iteration count and tape indices must
be equal; values within 1e-12 relative (tape values 1e-9).  Both then
postprocess one seeded reduced point, and the recovered x, y, z must agree
within 1e-12 relative.  The CPU oracle is left out here (about three minutes
at this size); it is compared with the reference on the smaller cases.
"""
import pytest

from gpp_b200 import lpgen
from test_reference_parity import ALL, check_against_reference, needs_reference

pytestmark = pytest.mark.gpu

BENCH = {"enable_folding": 1, "enable_structure_specific_rules": 1}


@needs_reference
def test_scale_lp_matches_reference():
    lp = lpgen.workload("scale", seed=0)
    got = check_against_reference(lp, ALL, BENCH, oracle=False, postsolve=True)
    m = got.ref["meta"]
    assert got.summary.folding_applied == int(m["folding_applied"])
    assert 13 in got.tape_types.tolist()   # the doubleton batch ran at scale
    assert got.summary.reduced_nnz < 0.8 * lp.nnz


@needs_reference
def test_qap30_matches_reference():
    lp = lpgen.workload("qap30", seed=0)
    assert (lp.m, lp.n) == (1_674_960, 810_900)
    got = check_against_reference(lp, ALL, BENCH, oracle=False, postsolve=True)
    m = got.ref["meta"]
    assert got.summary.folding_applied == int(m["folding_applied"])
    assert (got.summary.folded_rows, got.summary.folded_cols) == (int(m["folded_rows"]), int(m["folded_cols"]))
