# Builds the reference's MPS reader (plain C++, no CUDA) from its sources with
# a small driver that dumps the parsed arrays: the parity oracle of the
# engine's reader.  Usage: make -f oracle/mps_ref.mk  (from the repository root)
# Input: the reference checkout, from GPP_REFERENCE (environment) or
# REFERENCE=... on the command line; without one the recipe does nothing.
# Outputs only under oracle/_ref/.
REFERENCE ?= $(GPP_REFERENCE)
ifeq ($(wildcard $(REFERENCE)/cpp/mps_reader),)
all:
	@echo "$(lastword $(MAKEFILE_LIST)): no reference checkout (set GPP_REFERENCE); skipped"
else
OUT := oracle/_ref
CXX ?= g++
SRC := $(REFERENCE)/cpp/mps_reader/src/io/mpsreader.cpp \
       $(REFERENCE)/cpp/mps_reader/src/core/lp_model.cpp \
       $(REFERENCE)/cpp/mps_reader/src/core/sparse_matrix.cpp

all: $(OUT)/mps_ref_driver

$(OUT)/mps_ref_driver: oracle/mps_ref_driver.cpp $(SRC)
	@mkdir -p $(OUT)
	$(CXX) -std=c++17 -O2 -I$(REFERENCE)/cpp/mps_reader/include -o $@ oracle/mps_ref_driver.cpp $(SRC)
endif
