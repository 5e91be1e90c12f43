# Builds the upstream dip-fmm reference (C++20 core + its CUDA translation
# unit, which is needed only to satisfy the link: the CPU-only stub in the
# upstream tree lacks the FP32 overloads) from its sources where they lie,
# with every output written under oracle/_ref/.  This is test and baseline
# infrastructure: nothing in the product links or loads these files.
#
#   make -f oracle/ref.mk REF=/path/to/dip-fmm        (from the repo root; the default
#                                                      is a `reference` checkout beside the repo)
#
# Outputs
#   oracle/_ref/libcdfmm_ref.so   reference core (CpuStatic/CpuReference) + cuda_fmm.cu
#   oracle/_ref/ref_bench         CpuStatic timing/evaluation driver (oracle/ref_bench.cpp)
#   oracle/_ref/cdfmm*.so         the reference's own pybind11 module (golden-vector
#                                 generation in tests/golden/make_golden.py)
#
# The CPU code is compiled with the reference's Release intent (-O3, OpenMP),
# but -march=x86-64-v3 instead of -march=native because the binaries are built
# here and run on another host's CPU.

REF      ?= $(abspath ../reference)
OUT      := oracle/_ref
CUDA     ?= /usr/local/cuda
HOSTCXX  ?= /usr/bin/g++
NVCC     ?= $(CUDA)/bin/nvcc
PY       ?= python
PYINC    := $(shell $(PY) -c "import sysconfig;print(sysconfig.get_paths()['include'])")
PYBIND   := $(shell $(PY) -c "import pybind11;print(pybind11.get_include())")
PYEXT    := $(shell $(PY) -c "import sysconfig;print(sysconfig.get_config_var('EXT_SUFFIX'))")

CORE     := taylor_jet laplace_derivatives operators cuboid static_operators \
            validation uniform_tree uniform_fmm far_field near_field parameter_selection
DEFS     := -DCDFMM_USE_OPENMP=1 -DCDFMM_ENABLE_CUDA=1
CXXFLAGS := -std=c++20 -O3 -march=x86-64-v3 -fopenmp -fPIC $(DEFS) -I$(REF)/include -I$(REF)/src
NVFLAGS  := -std=c++20 -O3 -gencode arch=compute_100a,code=sm_100a $(DEFS) \
            -Xcompiler -fPIC -I$(REF)/include -I$(REF)/src
LDCUDA   := -L$(CUDA)/lib64 -Wl,-rpath,$(CUDA)/lib64 -lcudart -lcublas -lcusparse

OBJS     := $(addprefix $(OUT)/,$(addsuffix .o,$(CORE))) $(OUT)/cuda_fmm.o

all: $(OUT)/libcdfmm_ref.so $(OUT)/ref_bench $(OUT)/cdfmm$(PYEXT)

$(OUT):
	mkdir -p $(OUT)

$(OUT)/%.o: $(REF)/src/%.cpp | $(OUT)
	$(HOSTCXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/cuda_fmm.o: $(REF)/src/cuda_fmm.cu | $(OUT)
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OUT)/libcdfmm_ref.so: $(OBJS)
	$(HOSTCXX) -shared -fopenmp -o $@ $(OBJS) $(LDCUDA)

$(OUT)/ref_bench: oracle/ref_bench.cpp $(OUT)/libcdfmm_ref.so
	$(HOSTCXX) $(CXXFLAGS) -o $@ $< -L$(OUT) -Wl,-rpath,'$$ORIGIN' -lcdfmm_ref $(LDCUDA)

$(OUT)/cdfmm$(PYEXT): $(REF)/python/bindings.cpp $(OUT)/libcdfmm_ref.so
	$(HOSTCXX) $(CXXFLAGS) -shared -I$(PYINC) -I$(PYBIND) -o $@ $< \
	    -L$(OUT) -Wl,-rpath,'$$ORIGIN' -lcdfmm_ref $(LDCUDA)

.PHONY: all
