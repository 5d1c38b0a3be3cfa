# Builds the reference GPU-Preprocessor library (the bit-exact structure
# oracle, run only on a CUDA machine) straight from its sources with nvcc.
# Usage: make -f oracle/ref.mk -j8   (from the repository root)
# Input: the reference checkout, from GPP_REFERENCE (environment) or
# REFERENCE=... on the command line; without one the recipe does nothing.
# Outputs only under oracle/_ref/.
REFERENCE ?= $(GPP_REFERENCE)
ifeq ($(wildcard $(REFERENCE)/cpp/src),)
all:
	@echo "$(lastword $(MAKEFILE_LIST)): no reference checkout (set GPP_REFERENCE); skipped"
else
OUT := oracle/_ref
OBJ := $(OUT)/obj
NVCC ?= nvcc
ARCH ?= -gencode arch=compute_100,code=sm_100
NVFLAGS := -std=c++17 -O3 -rdc=true -Xcompiler -fPIC $(ARCH) \
           -DGPUPREPROCESSOR_USE_INT64_NNZ=0 -I$(REFERENCE)/cpp/include -w
SRC_DIR := $(REFERENCE)/cpp/src
SOURCES := \
  model/lp_problem.cpp folding/folding.cu folding/folding_kernels.cu \
  folding/folding_map.cu folding/folding_reduce.cu folding/folding_refinement.cu \
  presolve/transpose64.cu presolve/device_recovery.cu presolve/identity_plan.cu \
  presolve/fixed_variable_tape.cu presolve/gpu_postsolve.cu \
  presolve/postsolve/postsolve_piecewise_linear_reformulation_absolute_value.cu \
  presolve/postsolve/postsolve_piecewise_linear_reformulation_variable_pair.cu \
  presolve/gpu_presolve.cu presolve/gpu_presolve_kernels.cu presolve/presolve_structs.cu \
  presolve/rules/piecewise_linear_reformulation_variable_pair/shifted_antipodal.cu \
  presolve/rules/rule_two_row_variable_elimination.cu presolve/rules/rule_column_domination.cu \
  presolve/rules/rule_infeasible_and_fixed_variables.cu \
  presolve/rules/rule_infeasible_and_redundant_rows.cu presolve/rules/rule_doubleton_equations.cu \
  presolve/rules/rule_dual_fix.cu presolve/rules/empty_rows_and_columns/columns.cu \
  presolve/rules/empty_rows_and_columns/rows.cu \
  presolve/rules/rule_piecewise_linear_reformulation_variable_pair.cu \
  presolve/rules/piecewise_linear_reformulation_variable_pair/epigraph.cu \
  presolve/rules/rule_parallel_columns.cu presolve/rules/rule_parallel_rows.cu \
  presolve/rules/rule_zero_cost_product_variables.cu presolve/rules/rule_bound_strengthening.cu \
  presolve/rules/rule_redundant_variable_bounds.cu presolve/rules/rule_singleton_columns.cu \
  presolve/rules/rule_singleton_rows.cu \
  presolve/rules/rule_piecewise_linear_reformulation_absolute_value.cu
OBJECTS := $(addprefix $(OBJ)/,$(addsuffix .o,$(subst /,__,$(SOURCES))))

all: $(OUT)/libgpp_ref.so $(OUT)/ref_driver

$(OBJ)/%.o:
	@mkdir -p $(OBJ)
	$(NVCC) $(NVFLAGS) -x cu -c $(SRC_DIR)/$(subst __,/,$(basename $(notdir $@))) -o $@

$(OUT)/libgpp_ref.so: $(OBJECTS)
	$(NVCC) -shared $(ARCH) -Xcompiler -fPIC $(OBJECTS) -lcusparse -o $@

$(OUT)/ref_driver: oracle/ref_driver.cpp $(OUT)/libgpp_ref.so
	$(NVCC) -std=c++17 -O2 $(ARCH) -I$(REFERENCE)/cpp/include -Xcompiler -fPIC \
	  oracle/ref_driver.cpp -L$(OUT) -lgpp_ref -lcusparse -Xlinker -rpath,'$$ORIGIN' -o $@

.PHONY: all
endif
