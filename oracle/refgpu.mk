# Test infrastructure only: HornSculpt's own CudaBemSolver (the reference's GPU
# implementation of this path) compiled from the reference sources where they
# lie, with hornsculpt_b200/adapter/adapter_solve.cpp as its caller, into
# oracle/_ref/reference_solve. Same driver, same input format as the adapter
# over this library, so the two implementations run the same request.
#   make -f oracle/refgpu.mk REFERENCE=<reference root> -j8
REFERENCE ?=
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
ROOT := $(abspath $(HERE)/..)
OUT := $(HERE)_ref/refgpu
NVCC ?= nvcc
CXX ?= g++
INC := $(foreach d,$(wildcard $(REFERENCE)/modules/*/include),-I$(d)) -I$(REFERENCE)/modules/bem \
       -I$(REFERENCE)/modules/meshing/src -I$(REFERENCE)/modules/bem/cuda
CXXFLAGS := -std=c++20 -O2 -fPIC -w $(INC)
NVFLAGS := -std=c++20 -O3 -gencode arch=compute_100a,code=sm_100a -w $(INC) -Xcompiler -fPIC --expt-relaxed-constexpr

CU := $(wildcard $(REFERENCE)/modules/bem/cuda/*.cu)
CPP := $(wildcard $(REFERENCE)/modules/bem/*.cpp) $(wildcard $(REFERENCE)/modules/bem/galerkin/*.cpp) \
       $(wildcard $(REFERENCE)/modules/bem/fmm/*.cpp) $(wildcard $(REFERENCE)/modules/lem/src/*.cpp) \
       $(REFERENCE)/modules/meshing/src/mesh_quality.cpp $(REFERENCE)/modules/meshing/src/acoustic_partition.cpp \
       $(REFERENCE)/modules/meshing/src/symmetry_sector.cpp
OBJ := $(patsubst $(REFERENCE)/%.cu,$(OUT)/%.o,$(CU)) $(patsubst $(REFERENCE)/%.cpp,$(OUT)/%.o,$(CPP))

$(HERE)_ref/reference_solve: $(OBJ) $(HERE)ref_gpu_stubs.cpp $(ROOT)/hornsculpt_b200/adapter/adapter_solve.cpp
	$(NVCC) -std=c++20 -O2 -gencode arch=compute_100a,code=sm_100a $(INC) -w -o $@ $(OBJ) \
	  $(HERE)ref_gpu_stubs.cpp $(ROOT)/hornsculpt_b200/adapter/adapter_solve.cpp -lcublas -lcusolver -lcufft -lpthread

$(OUT)/%.o: $(REFERENCE)/%.cu
	@mkdir -p $(dir $@)
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OUT)/%.o: $(REFERENCE)/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -c $< -o $@
