"""Small hand-built LPs and a runner that presolves them on either backend.

The cases re-express the reference's rule-level known-answer tests
(cpp/tests/test_rule_*.cpp) as whole-pipeline runs with only the rule under
test enabled; where a reference case sets up a plan state by hand (an already
removed column, say), the LP here reaches that state through an earlier rule
of the same cleanup pass, and the comment at the case says how.
"""
import numpy as np

from gpp_b200 import lpgen
from gpp_b200.capi import params_with_rules

INF = np.inf


def make_lp(n, rows, c, l, u, AL, AU):
    """rows: list of [(col, value), ...] in stored order."""
    ptr = [0]
    idx, val = [], []
    for r in rows:
        for j, a in r:
            idx.append(j)
            val.append(a)
        ptr.append(len(idx))
    lp = lpgen.HostLP(len(rows), n, np.array(ptr, np.int32), np.array(idx, np.int32), np.array(val, np.float64),
                      np.array(c, np.float64), np.array(AL, np.float64), np.array(AU, np.float64),
                      np.array(l, np.float64), np.array(u, np.float64))
    return lp.ensure_transpose()


class Run:
    """Presolve `lp` with `rules` on 'oracle' or 'gpu' and keep host copies."""

    def __init__(self, backend, lp, rules, **extra):
        extra.setdefault("enable_folding", 0)
        params = params_with_rules(rules, **extra)
        if backend == "oracle":
            import pyoracle
            self.r = pyoracle.presolve(lp, params)
            self.fold = self.r.fold_map()
        else:
            from gpp_b200 import device
            dlp = device.DeviceLp(lp)
            s = device.preprocess(dlp, params)
            try:
                self.r = device.Result(s)
                self.fold = device.fold_map(s)
                self.r.summary = type(s).from_buffer_copy(s)   # free_summary clears s
            finally:
                device.free_summary(s)
        self.s = self.r.summary

    def record(self, k):
        r = self.r
        return (int(r.tape_types[k]), r.tape_idx[r.tape_is[k]:r.tape_is[k + 1]].tolist(),
                r.tape_val[r.tape_vs[k]:r.tape_vs[k + 1]])

    def __getattr__(self, name):
        return getattr(self.r, name)


def bits(x):
    return np.asarray(x, np.float64).view(np.uint64)
