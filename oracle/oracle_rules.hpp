// Oracle rule declarations.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#pragma once
#include "oracle.hpp"

namespace oracle {
void refresh_stats(Stats& s, const Lp& lp, const Plan& plan);
void rule_fixed_variables(Plan& plan, const Lp& lp, const gpp_params& p);
void rule_empty_columns(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_empty_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_singleton_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_singleton_columns(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_bound_strengthening(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_redundant_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_dual_fix(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_column_domination(Plan& plan, const Lp& lp, const gpp_params& p);
void rule_two_row_variable_elimination(Plan& plan, const Lp& lp, const gpp_params& p);
void rule_zero_cost_product_variables(Plan& plan, const Lp& lp, const gpp_params& p);
void rule_parallel_rows(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_parallel_columns(Plan& plan, const Lp& lp, const Stats& s, const gpp_params& p);
void rule_doubleton_equations(Plan& plan, const Lp& lp, const gpp_params& p);
}  // namespace oracle
