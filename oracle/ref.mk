# Recipe for the compiled reference checker (test infrastructure only).
# Builds, from the reference sources where they lie, into oracle/_ref/:
#   cloth_bag      the reference FP64 CPU cloth executable (tools/cloth_bag.cpp)
#   libref_shim.so the same source behind the C API of ref_shim.cpp
#   cloth_calibration the reference calibration qualifier (tools/cloth_calibration.cpp)
# Nothing here is copied into the repository; _ref/ is git-ignored.
# the reference checkout: NUMI_CLOTH_REFERENCE, default /root/reference
NUMI_CLOTH_REFERENCE ?= /root/reference
REFERENCE ?= $(NUMI_CLOTH_REFERENCE)
CXX ?= g++
HERE := $(abspath $(dir $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)/_ref
FLAGS := -std=c++23 -O3 -I$(REFERENCE)/include -I$(REFERENCE)

all: $(OUT)/cloth_bag $(OUT)/libref_shim.so $(OUT)/cloth_calibration

$(OUT)/cloth_bag: $(REFERENCE)/tools/cloth_bag.cpp
	@mkdir -p $(OUT)
	$(CXX) $(FLAGS) $< -o $@

$(OUT)/cloth_calibration: $(REFERENCE)/tools/cloth_calibration.cpp
	@mkdir -p $(OUT)
	$(CXX) $(FLAGS) $< -o $@

# Linked against the shared libstdc++ so that it can share a process with
# Python extension modules that already loaded it.
LIBSTDCXX ?= $(shell $(CXX) -print-file-name=libstdc++.so.6)

$(OUT)/libref_shim.so: $(HERE)/ref_shim.cpp $(HERE)/oracle.h $(REFERENCE)/tools/cloth_bag.cpp
	@mkdir -p $(OUT)
	$(CXX) $(FLAGS) -I$(HERE) -fPIC -shared $(HERE)/ref_shim.cpp $(LIBSTDCXX) -o $@

.PHONY: all
