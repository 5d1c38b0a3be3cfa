"""ctypes mirror of include/gpp.h and the loader of the CUDA engine.

The engine is the shared library ``libgpp_b200.so`` built in this directory by
``build.py`` (sm_100a).  ``load()`` fails loudly when it is missing: there is
no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpp_b200.so")

u8, i32, i64, f64 = C.c_uint8, C.c_int32, C.c_int64, C.c_double
P = C.POINTER


class Csr(C.Structure):
    _fields_ = [("rows", i32), ("cols", i32), ("nnz", i32),
                ("rowPtr", C.c_void_p), ("colVal", C.c_void_p), ("nzVal", C.c_void_p)]


class Lp(C.Structure):
    _fields_ = [("A", Csr), ("AT", Csr), ("c", C.c_void_p), ("AL", C.c_void_p),
                ("AU", C.c_void_p), ("l", C.c_void_p), ("u", C.c_void_p),
                ("obj_constant", f64), ("AT_leading_slack", i32), ("AT_slack_after", C.c_void_p)]


_PARAM_FIELDS = [
    ("max_iters", i32, 512), ("max_time", f64, math.inf), ("verbose", u8, 0),
    ("record_postsolve_tape", u8, 1), ("record_postsolve_tape_cpu", u8, 0),
    ("enable_presolve", u8, 1), ("enable_folding", u8, 1), ("folding_tolerance", f64, 1e-8),
    ("feasibility_tol", f64, 1e-6), ("bound_tol", f64, 1e-6), ("zero_tol", f64, 1e-10),
    ("bound_strengthening_upper_relaxation_factor", f64, 1.0),
    ("bound_strengthening_max_rounds", i32, 64),
    ("bound_strengthening_max_bound_only_rounds", i32, 64),
    ("bound_strengthening_preserve_free_zero_cost", u8, 1),
    ("doubleton_equations_max_fill_in_proxy", i32, 96), ("doubleton_equations_scan", u8, 1),
    ("doubleton_equations_min_selected_per_batch", i32, 256),
    ("doubleton_equations_min_selected_ratio", f64, 0.005),
    ("doubleton_equations_max_batch_rounds", i32, 0), ("doubleton_equations_max_time", f64, 0.0),
    ("enable_infeasible_and_fixed_variables", u8, 1), ("enable_empty_rows", u8, 1),
    ("enable_singleton_rows", u8, 1), ("enable_infeasible_and_redundant_rows", u8, 1),
    ("enable_bound_strengthening", u8, 1), ("enable_parallel_rows", u8, 1),
    ("enable_empty_columns", u8, 1), ("enable_singleton_columns", u8, 1),
    ("enable_doubleton_equations", u8, 1), ("enable_dual_fix", u8, 1),
    ("dual_fix_max_nonzero_cost_col_degree", i32, 128), ("enable_parallel_columns", u8, 1),
    ("parallel_columns_max_abs_ratio", f64, 2.0),
    ("parallel_columns_scale_guard_max_group_size", i32, 4),
    ("parallel_columns_scale_guard_min_groups", i32, 128),
    ("enable_structure_specific_rules", u8, 1),
    ("enable_two_row_variable_elimination", u8, 1),
    ("two_row_variable_elimination_max_row_nnz", i32, 8),
    ("two_row_variable_elimination_safety_tol", f64, 1.0e-8),
    ("two_row_variable_elimination_min_candidates", i32, 128),
    ("two_row_variable_elimination_min_candidate_ratio", f64, 0.01),
    ("enable_zero_cost_product_variables", u8, 1),
    ("zero_cost_product_variables_min_candidates", i32, 128),
    ("zero_cost_product_variables_min_candidate_ratio", f64, 0.01),
    ("enable_piecewise_linear_reformulation_variable_pair", u8, 1),
    ("piecewise_linear_reformulation_variable_pair_epigraph_probe_pairs", i32, 256),
    ("piecewise_linear_reformulation_variable_pair_epigraph_min_pairs", i32, 4096),
    ("piecewise_linear_reformulation_variable_pair_epigraph_min_potential_gain", f64, 0.20),
    ("piecewise_linear_reformulation_variable_pair_epigraph_min_actual_gain", f64, 0.20),
    ("piecewise_linear_reformulation_variable_pair_epigraph_max_tail_cols", i32, 8),
    ("piecewise_linear_reformulation_variable_pair_epigraph_max_quotient_terms_per_row", i32, 5),
    ("piecewise_linear_reformulation_variable_pair_shifted_antipodal_probe_pairs", i32, 256),
    ("piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_pairs", i32, 4096),
    ("piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_potential_gain", f64, 0.20),
    ("piecewise_linear_reformulation_variable_pair_shifted_antipodal_min_actual_gain", f64, 0.20),
    ("piecewise_linear_reformulation_variable_pair_shifted_antipodal_max_quotient_terms_per_row", i32, 6),
    ("enable_column_domination", u8, 1),
    ("column_domination_probe_rows", i32, 64),
    ("column_domination_probe_cols", i32, 256),
    ("column_domination_probe_nnz", i32, 256),
    ("column_domination_min_fixed_cols", i32, 4096),
    ("column_domination_min_candidate_ratio", f64, 0.20),
    ("enable_piecewise_linear_reformulation_absolute_value", u8, 1),
    ("piecewise_linear_reformulation_absolute_value_residual_bound_mode", u8, 0),
    ("piecewise_linear_reformulation_absolute_value_residual_bound_as_free_min", f64, 1.0e8),
    ("enable_redundant_variable_bounds", u8, 0),
    ("enable_startup", u8, 1),
    ("bound_strengthening_bound_only_nnz_round_budget", i64, 8000000),
]


class Params(C.Structure):
    _fields_ = [(name, typ) for name, typ, _ in _PARAM_FIELDS]

    @classmethod
    def defaults(cls, **overrides) -> "Params":
        p = cls()
        for name, _, value in _PARAM_FIELDS:
            setattr(p, name, value)
        for k, v in overrides.items():
            if not hasattr(p, k):
                raise AttributeError(k)
            setattr(p, k, v)
        return p


RULE_FLAGS = ["enable_infeasible_and_fixed_variables", "enable_empty_rows", "enable_singleton_rows",
              "enable_infeasible_and_redundant_rows", "enable_bound_strengthening",
              "enable_parallel_rows", "enable_empty_columns", "enable_singleton_columns",
              "enable_doubleton_equations", "enable_dual_fix", "enable_parallel_columns"]


def params_with_rules(rules, **extra) -> Params:
    """Parameters with exactly the named rules enabled (names without 'enable_')."""
    kw = {f: 0 for f in RULE_FLAGS}
    for r in rules:
        kw["enable_" + r] = 1
    kw.update(extra)
    return Params.defaults(**kw)


class Summary(C.Structure):
    _fields_ = [("original_rows", i32), ("original_cols", i32), ("reduced_rows", i32),
                ("reduced_cols", i32), ("reduced_nnz", i32), ("iterations", i32),
                ("stopped_at_iteration_limit", u8), ("has_change", u8), ("has_infeasible", u8),
                ("has_unbounded", u8), ("presolve_enabled", u8), ("folding_applied", u8),
                ("owns_reduced_lp", u8), ("elapsed_seconds", f64), ("preprocessing_seconds", f64),
                ("obj_constant_delta", f64), ("reduced_lp", Lp), ("record", C.c_void_p),
                ("folded_rows", i32), ("folded_cols", i32)]


class HostLp(C.Structure):
    """gpp_host_lp: A as a host CSR and the vectors (host pointers)."""
    _fields_ = [("rows", i32), ("cols", i32), ("nnz", i32), ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p),
                ("val", C.c_void_p), ("c", C.c_void_p), ("AL", C.c_void_p), ("AU", C.c_void_p),
                ("l", C.c_void_p), ("u", C.c_void_p), ("obj_constant", f64)]


class AbsoluteValueRecovery(C.Structure):
    """gpp_absolute_value_recovery: one step as host arrays (pointers)."""
    _fields_ = [("pattern", i32), ("split_count", i32), ("split_t", C.c_void_p), ("split_e", C.c_void_p),
                ("split_rho", C.c_void_p), ("pair_count", i32), ("pair_bound", C.c_void_p),
                ("pair_free", C.c_void_p), ("linked_count", i32), ("linked_slack", C.c_void_p),
                ("linked_t", C.c_void_p), ("linked_factor", C.c_void_p), ("max_group_count", i32),
                ("max_slack", C.c_void_p), ("max_starts", C.c_void_p), ("max_t", C.c_void_p),
                ("max_factor", C.c_void_p)]


_lib = None


def load():
    """Load the engine library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA engine not built: {LIB_PATH} is missing (run build.py)")
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "gpp_default_params": (None, [P(Params)]),
        "gpp_preprocess": (C.c_int, [P(Lp), P(Params), P(Summary)]),
        "gpp_run_presolve": (C.c_int, [P(Lp), P(Params), C.c_int, P(Summary)]),
        "gpp_postprocess": (C.c_int, [vp, vp, vp, P(Summary), P(Lp), vp, vp, vp]),
        "gpp_postsolve_device": (C.c_int, [vp, vp, vp, P(Summary), P(Lp), vp, vp, vp]),
        "gpp_postsolve_device_lower": (C.c_int, [vp, vp, vp, P(Summary), P(Lp), vp, vp, vp, vp]),
        "gpp_free_summary": (None, [P(Summary)]),
        "gpp_export_maps": (C.c_int, [P(Summary), vp, vp]),
        "gpp_tape_sizes": (C.c_int, [P(Summary), P(i64), P(i64), P(i64), P(i64)]),
        "gpp_export_tape": (C.c_int, [P(Summary), vp, vp, vp, vp, vp, vp, vp]),
        "gpp_row_activity_summary": (C.c_int, [P(Csr), vp, vp, f64, vp, vp, vp, vp, vp, vp, vp]),
        "gpp_live_stats": (C.c_int, [P(Csr), vp, vp, vp, vp, vp, vp, vp, vp]),
        "gpp_col_max_abs": (C.c_int, [P(Csr), vp, vp]),
        "gpp_compact_and_transpose": (C.c_int, [P(Csr), vp, vp, P(Csr), P(Csr)]),
        "gpp_parallel_row_hashes": (C.c_int, [P(Csr), vp, vp, C.c_int, vp]),
        "gpp_sort_pairs": (C.c_int, [vp, vp, i64]),
        "gpp_sort_pairs_static": (C.c_int, [vp, vp, i64, vp]),
        "gpp_export_folding_map": (C.c_int, [C.POINTER(Summary), vp, vp, vp, vp]),
        "gpp_unfold_solution": (C.c_int, [C.POINTER(Summary), vp, vp, vp, vp, vp, vp]),
        "gpp_device_alloc": (C.c_int, [C.POINTER(vp), C.c_size_t]),
        "gpp_device_free": (None, [vp]),
        "gpp_last_error": (C.c_char_p, []),
        "gpp_kernel_launches": (C.c_uint64, [C.c_int]),
        "gpp_host_syncs": (C.c_uint64, [C.c_int]),
        "gpp_preprocess_batch": (C.c_int, [vp, C.c_int32, P(Params), C.c_int32, vp, vp]),
        "gpp_preprocess_traced": (C.c_int, [P(Lp), P(Params), P(Summary), vp, vp, vp, C.c_int32, P(C.c_int32)]),
        "gpp_mps_read": (C.c_int, [C.c_char_p, P(vp)]),
        "gpp_mps_read_string": (C.c_int, [C.c_char_p, P(vp)]),
        "gpp_mps_info": (C.c_int, [vp, P(C.c_int32), P(C.c_int32), P(i64), P(f64), C.c_char_p, C.c_size_t]),
        "gpp_mps_arrays": (C.c_int, [vp] + [vp] * 11),
        "gpp_mps_free": (None, [vp]),
        "gpp_mps_upload": (C.c_int, [vp, P(Lp)]),
        "gpp_lp_free": (None, [P(Lp)]),
        "gpp_lp_from_host": (C.c_int, [P(HostLp), P(Lp)]),
        "gpp_export_reduced": (C.c_int, [P(Summary), C.c_char_p, C.c_char_p]),
        "gpp_reduced_to_device": (C.c_int, [P(Summary), P(Lp)]),
        "gpp_reduced_to_host": (C.c_int, [P(Summary)] + [vp] * 9),
        "gpp_schedule_model_create": (C.c_int, [vp, C.c_double, C.c_double, P(vp)]),
        "gpp_schedule_model_free": (None, [vp]),
        "gpp_schedule_model_create_per_rule": (C.c_int, [vp, vp, C.c_double, P(vp)]),
        "gpp_preprocess_scheduled": (C.c_int, [P(Lp), P(Params), vp, P(Summary)]),
        "gpp_mlp_train": (C.c_int, [vp, vp, vp, vp, i64, C.c_int32, C.c_int32, C.c_float, C.c_uint64, vp]),
        "gpp_mlp_forward": (C.c_int, [vp, vp, i64, vp]),
        "gpp_mlp_gradients": (C.c_int, [vp, vp, vp, vp, i64, vp, vp]),
        "gpp_postprocess_batch": (C.c_int, [vp, vp, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp]),
        "gpp_batch_autotune": (C.c_int, [vp, C.c_int32, P(Params), C.c_int32, P(C.c_int32), vp]),
        "gpp_profile_enable": (None, [C.c_int]),
        "gpp_profile_read": (C.c_int, [C.c_int, C.c_char_p, C.c_size_t, P(i64), P(f64), P(f64)]),
        "gpp_inject_alloc_failure": (None, [i64]),
        "gpp_recovery_checkpoints": (C.c_int, [P(Summary), P(i32), vp, vp, vp]),
        "gpp_absolute_value_sizes": (C.c_int, [P(Summary), i32, vp]),
        "gpp_export_absolute_value": (C.c_int, [P(Summary), i32] + [vp] * 12),
        "gpp_restore_absolute_value": (C.c_int, [vp, P(AbsoluteValueRecovery), i32, vp]),
        "gpp_variable_pair_size": (C.c_int, [P(Summary), i32, P(i32)]),
        "gpp_export_variable_pair": (C.c_int, [P(Summary), i32] + [vp] * 6),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


EXPORTED = [
    "gpp_default_params", "gpp_preprocess", "gpp_run_presolve", "gpp_postprocess",
    "gpp_postsolve_device", "gpp_free_summary", "gpp_export_maps", "gpp_tape_sizes",
    "gpp_export_tape", "gpp_row_activity_summary", "gpp_live_stats", "gpp_col_max_abs",
    "gpp_compact_and_transpose", "gpp_parallel_row_hashes", "gpp_sort_pairs", "gpp_sort_pairs_static", "gpp_device_alloc", "gpp_device_free",
    "gpp_export_folding_map", "gpp_unfold_solution", "gpp_run_folding", "gpp_free_folding_run",
    "gpp_folding_run_export_map", "gpp_folding_run_unfold", "gpp_inject_alloc_failure",
    "gpp_last_error", "gpp_kernel_launches", "gpp_host_syncs",
    "gpp_preprocess_batch", "gpp_postprocess_batch", "gpp_batch_autotune",
    "gpp_mps_read", "gpp_mps_read_string", "gpp_mps_info", "gpp_mps_arrays", "gpp_mps_free", "gpp_mps_upload",
    "gpp_lp_free", "gpp_lp_from_host", "gpp_export_reduced", "gpp_reduced_to_device", "gpp_reduced_to_host",
    "gpp_preprocess_traced", "gpp_schedule_model_create", "gpp_schedule_model_free",
    "gpp_schedule_model_create_per_rule", "gpp_preprocess_scheduled",
    "gpp_mlp_train", "gpp_mlp_forward", "gpp_mlp_gradients", "gpp_profile_enable", "gpp_profile_read",
    "gpp_recovery_checkpoints", "gpp_absolute_value_sizes", "gpp_export_absolute_value", "gpp_postsolve_device_lower",
    "gpp_restore_absolute_value", "gpp_variable_pair_size", "gpp_export_variable_pair",
]

# Absolute-value recovery patterns (include/gpp.h GPP_ABS_*).
ABS_L1_SPLIT, ABS_GRAPH_L1, ABS_OUTER_PAIR = 1, 2, 3


def check(status: int) -> None:
    if status != 0:
        msg = load().gpp_last_error().decode(errors="replace")
        raise RuntimeError(f"gpp error {status}: {msg}")


def profile_read():
    """Per-kernel (name, launches, ms, bytes) recorded since gpp_profile_enable(1)."""
    lib = load()
    out = []
    count = lib.gpp_profile_read(0, None, 0, None, None, None)
    for k in range(max(count, 0)):
        name = C.create_string_buffer(128)
        launches, ms, by = i64(), f64(), f64()
        lib.gpp_profile_read(k, name, 128, C.byref(launches), C.byref(ms), C.byref(by))
        out.append((name.value.decode(), launches.value, ms.value, by.value))
    return out
