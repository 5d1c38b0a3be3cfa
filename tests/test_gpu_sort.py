"""The engine's stable radix sort of (hash, index) pairs against numpy."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_radix_sort_pairs_matches_numpy():
    import torch
    from gpp_b200 import capi
    lib = capi.load()
    rng = np.random.default_rng(0)
    # Up to 4096 pairs one block sorts them; above, the radix passes do.
    for n in (1, 3, 7, 2048, 2049, 4096, 4097, 100_003):
        keys = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
        keys[rng.random(n) < 0.3] = keys[0]        # many duplicates: stability matters
        keys[: n // 10] &= np.uint64(0xFFFF)        # some small keys: skipped passes
        keys[rng.random(n) < 0.05] |= np.uint64(1 << 63)   # unsigned order
        vals = (np.arange(n, dtype=np.int32) * 7919) % max(n, 1)
        dk = torch.from_numpy(keys.view(np.int64)).cuda()
        dv = torch.from_numpy(vals).cuda()
        assert lib.gpp_sort_pairs(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n) == 0
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
        assert np.array_equal(dv.cpu().numpy(), vals[order])
