"""The C-ABI library builds, loads and exports every entry point that
include/gpp.h declares; without a device every compute entry point fails
loudly (there is no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

from gpp_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gpp.h")).read()
    return sorted(set(re.findall(r"GPP_API\s+[\w\s\*]+?\b(gpp_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(capi.EXPORTED) == names


def test_default_params_match_reference_defaults():
    lib = capi.load()
    p = capi.Params()
    lib.gpp_default_params(C.byref(p))
    q = capi.Params.defaults()
    assert bytes(p) == bytes(q)
    assert p.max_iters == 512 and p.feasibility_tol == 1e-6 and p.zero_tol == 1e-10
    assert p.doubleton_equations_min_selected_per_batch == 256
    assert p.bound_strengthening_bound_only_nnz_round_budget == 8_000_000


def test_free_summary_is_idempotent_on_empty():
    lib = capi.load()
    s = capi.Summary()
    lib.gpp_free_summary(C.byref(s))
    lib.gpp_free_summary(C.byref(s))
    assert s.record is None


def test_no_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    lib = capi.load()
    s = capi.Summary()
    lp = capi.Lp()
    p = capi.Params.defaults()
    st = lib.gpp_preprocess(C.byref(lp), C.byref(p), C.byref(s))
    assert st == 5
    assert b"no CUDA device" in lib.gpp_last_error()
    # Loading a host LP (A^T is built on the device) has no host fallback either.
    host = capi.HostLp()
    assert lib.gpp_lp_from_host(C.byref(host), C.byref(lp)) == 5
