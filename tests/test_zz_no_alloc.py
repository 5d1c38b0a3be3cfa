"""gpp_sort_pairs_static, the pair sort that allocates nothing, against the
pooled gpp_sort_pairs, both through the C ABI.

Two calls of the fixed-scratch sort in a row (the largest size it accepts,
then a smaller one over the same shared scratch) must return exactly what the
pooled sort returns; the second call must leave the device's free memory
unchanged; a size above the fixed capacity is refused with GPP_ERR_LENGTH and
leaves the data alone.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gpp_b200 import capi

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPP_ERR_LENGTH = 2


def max_pairs():
    text = open(os.path.join(ROOT, "include", "gpp.h")).read()
    return 1 << int(re.search(r"#define GPP_SORT_STATIC_MAX_PAIRS \(1 << (\d+)\)", text).group(1))


def make_pairs(rng, n):
    keys = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
    keys[rng.random(n) < 0.3] = keys[0]          # many duplicates: stability matters
    keys[: n // 10] &= np.uint64(0xFFFF)          # small keys: high digits constant
    vals = np.arange(n, dtype=np.int32)[::-1].copy()
    return keys, vals


def test_static_sort_matches_pooled_sort_on_two_calls_in_a_row():
    import torch
    lib = capi.load()
    rng = np.random.default_rng(7)
    stream = torch.cuda.current_stream()
    # An empty sort is the set-up call: it loads the array and looks up its address.
    assert lib.gpp_sort_pairs_static(None, None, 0, C.c_void_p(stream.cuda_stream)) == 0, lib.gpp_last_error()
    for call, n in enumerate((max_pairs(), 100_003)):
        keys, vals = make_pairs(rng, n)
        pk = torch.from_numpy(keys.view(np.int64)).cuda()
        pv = torch.from_numpy(vals).cuda()
        assert lib.gpp_sort_pairs(C.c_void_p(pk.data_ptr()), C.c_void_p(pv.data_ptr()), n) == 0
        sk = torch.from_numpy(keys.view(np.int64)).cuda()
        sv = torch.from_numpy(vals).cuda()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        status = lib.gpp_sort_pairs_static(C.c_void_p(sk.data_ptr()), C.c_void_p(sv.data_ptr()), n,
                                           C.c_void_p(stream.cuda_stream))
        assert status == 0, lib.gpp_last_error()
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
        assert torch.equal(sk, pk) and torch.equal(sv, pv)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(sk.cpu().numpy().view(np.uint64), keys[order])
        assert np.array_equal(sv.cpu().numpy(), vals[order])


def test_static_sort_refuses_sizes_above_its_capacity():
    import torch
    lib = capi.load()
    n = max_pairs() + 1
    keys = torch.arange(n, 0, -1, dtype=torch.int64, device="cuda")
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    status = lib.gpp_sort_pairs_static(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()), n, None)
    assert status == GPP_ERR_LENGTH
    assert b"capacity" in lib.gpp_last_error()
    torch.cuda.synchronize()
    assert torch.equal(keys, torch.arange(n, 0, -1, dtype=torch.int64, device="cuda"))
    # Trivial sizes are no-ops.
    assert lib.gpp_sort_pairs_static(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()), 1, None) == 0
    assert lib.gpp_sort_pairs_static(None, None, 0, None) == 0
