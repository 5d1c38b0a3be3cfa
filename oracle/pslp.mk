# Builds the reference's bundled CPU presolver (PSLP 0.0.11, the CPU baseline)
# from its sources, with the flags the reference's build uses, plus a small
# timing driver.  Usage: make -f oracle/pslp.mk   (from the repository root)
# Input: the reference checkout, from GPP_REFERENCE (environment) or
# REFERENCE=... on the command line; without one the recipe does nothing.
# Outputs only under oracle/_ref/.
REFERENCE ?= $(GPP_REFERENCE)
ifeq ($(wildcard $(REFERENCE)/third_party/pslp),)
all:
	@echo "$(lastword $(MAKEFILE_LIST)): no reference checkout (set GPP_REFERENCE); skipped"
else
PSLP := $(REFERENCE)/third_party/pslp
OUT := oracle/_ref
CC ?= gcc
CFLAGS := -O3 -std=c11 -DNDEBUG -D_POSIX_C_SOURCE=200809L -DPSLP_VERSION='"0.0.11"' -I$(PSLP)/include -I$(PSLP)/include/PSLP -I$(PSLP)/include/core -I$(PSLP)/include/data_structures -I$(PSLP)/include/explorers -w
SOURCES := $(wildcard $(PSLP)/src/core/*.c) $(wildcard $(PSLP)/src/explorers/*.c)

all: $(OUT)/pslp_driver

$(OUT)/pslp_driver: oracle/pslp_driver.c $(SOURCES)
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) oracle/pslp_driver.c $(SOURCES) -lm -lpthread -o $@
endif
