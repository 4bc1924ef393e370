# Builds the reference's own GPU code of DWGTech/DWG -- src/TurboDWG.cu,
# src/TurboLibiGWN.cu, src/TurboMC.cu, src/TurboNormalInit.cu and
# src/KNN_GWN.cu, unchanged, from the reference checkout -- plus the C shim of
# this directory into _ref/libref_dwg.so.  Test infrastructure only (a
# comparator for the GWN sums, marching cubes and the whole DWG loop).
#
# The reference's CMake build compiles these with "-O3 --use_fast_math"
# (CMakeLists.txt:77); the same flags are used here.  Its host signatures name
# a few Eigen types: ref_eigen/Eigen/Core is a small stand-in for exactly those
# names (Eigen itself is not installed).  Forced includes supply what the
# sources take from headers that are no longer transitive in CUDA 12.9:
# <cfloat> (FLT_MAX in cudaKDTree) and thrust's sequence/sort (TurboDWG.cu).
#
# Usage: make -f ref_dwg.mk [REF=<reference checkout>]; REF defaults to the
# DWG_REFERENCE environment variable.
REF ?= $(DWG_REFERENCE)
NVCC ?= /usr/local/cuda/bin/nvcc
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref/libref_dwg.so
OBJ := $(HERE)_ref/dwg
SRCS := TurboDWG TurboLibiGWN TurboMC TurboNormalInit KNN_GWN
FLAGS := -gencode arch=compute_100a,code=sm_100a -O3 --use_fast_math -std=c++17 -Xcompiler -fPIC \
         -include cfloat -include thrust/sequence.h -include thrust/sort.h \
         -I$(HERE)ref_eigen -I$(REF)/include -I$(REF)/include/cudaKDTree --expt-relaxed-constexpr -w

all: $(OUT)

$(OBJ)/%.o: $(REF)/src/%.cu
	@test -n "$(REF)" || (echo "set REF or DWG_REFERENCE to the reference checkout" && false)
	mkdir -p $(OBJ)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OBJ)/shim.o: $(HERE)ref_dwg_shim.cu $(HERE)ref_eigen/Eigen/Core
	mkdir -p $(OBJ)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT): $(foreach s,$(SRCS),$(OBJ)/$(s).o) $(OBJ)/shim.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -cudart static -o $@ $^

.PHONY: all
