# Builds the reference's GPU kNN (cudaKDTree builder + cct kNN of DWGTech/DWG,
# src/KNN_GWN.cu) from the reference sources in place, plus the C shim of this
# directory, into _ref/libref_knn.so.  Test infrastructure only (a comparator).
# Needs the reference checkout; the output is git-ignored and travels with the
# repository snapshot.  Usage: make -f ref_knn.mk REF=<reference checkout> (default: $DWG_REFERENCE)
REF ?= $(DWG_REFERENCE)
NVCC ?= /usr/local/cuda/bin/nvcc
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref/libref_knn.so
FLAGS := -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC -include cfloat \
         -I$(REF)/include -I$(REF)/include/cudaKDTree --expt-relaxed-constexpr -w

all: $(OUT)

$(OUT): $(REF)/src/KNN_GWN.cu $(HERE)ref_knn_shim.cu
	mkdir -p $(HERE)_ref
	$(NVCC) $(FLAGS) -c $(REF)/src/KNN_GWN.cu -o $(HERE)_ref/knn_gwn.o
	$(NVCC) $(FLAGS) -c $(HERE)ref_knn_shim.cu -o $(HERE)_ref/shim.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -cudart static -o $@ $(HERE)_ref/knn_gwn.o $(HERE)_ref/shim.o

.PHONY: all
