# oracle/ref.mk -- builds the REFERENCE (fGPE v0.3) from its own sources, where
# they lie, into oracle/_ref/ (git-ignored).  Test infrastructure only.
#
#   make -f oracle/ref.mk REF=/path/to/fGPE
#
# Outputs:
#   _ref/libref_host.so  the reference's host classes (InputVariables, Params,
#                        Params2, Psi, Vext, Output) + oracle/ref_host_shim.cpp.
#                        Pure host code: runs on any CPU; pins fgpe_b200/host.
#   _ref/gpe_ref         the stock reference binary (its main.cu + plugins),
#                        sm_100a, cuFFT.  Needs a GPU.
#   _ref/gpe_ref_trace   reference sources + oracle/ref_plugin_main.cu
#                        (constant-g / quench / template test plugins that log
#                        full-precision PARS).  Needs a GPU.
# The reference's own Makefile passes no -arch; here every object is built for
# sm_100a with the reference's other flags (-std=c++20 -O3).
# the reference's source tree: REF=..., else $GPE_REFERENCE_DIR, else /root/reference
GPE_REFERENCE_DIR ?= /root/reference
REF   ?= $(GPE_REFERENCE_DIR)
HERE  := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT   := $(HERE)_ref
OBJ   := $(OUT)/obj
NVCC  ?= nvcc
ARCH  := -gencode arch=compute_100a,code=sm_100a
FLAGS := -I$(REF)/hpp -I$(REF) -std=c++20 -O3 -Wno-deprecated-gpu-targets -diag-suppress 1650,2464,550,177,20012 $(ARCH)

HOST_SRCS := input_variables params params2 psi vext output
ALL_SRCS  := $(patsubst $(REF)/src/%.cu,%,$(wildcard $(REF)/src/*.cu))
HAM_SRCS  := $(patsubst $(REF)/hamiltonians/%.cu,%,$(wildcard $(REF)/hamiltonians/*.cu))

HOST_OBJS := $(addprefix $(OBJ)/pic_,$(addsuffix .o,$(HOST_SRCS)))
SRC_OBJS  := $(addprefix $(OBJ)/src_,$(addsuffix .o,$(ALL_SRCS)))
HAM_OBJS  := $(addprefix $(OBJ)/ham_,$(addsuffix .o,$(HAM_SRCS)))

all: $(OUT)/libref_host.so $(OUT)/gpe_ref $(OUT)/gpe_ref_trace
host: $(OUT)/libref_host.so

$(OBJ):
	mkdir -p $(OBJ)

$(OBJ)/pic_%.o: $(REF)/src/%.cu | $(OBJ)
	$(NVCC) $(FLAGS) -Xcompiler -fPIC -c $< -o $@

$(OBJ)/src_%.o: $(REF)/src/%.cu | $(OBJ)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OBJ)/ham_%.o: $(REF)/hamiltonians/%.cu | $(OBJ)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OBJ)/main.o: $(REF)/main.cu | $(OBJ)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OBJ)/shim.o: $(HERE)ref_host_shim.cpp | $(OBJ)
	$(NVCC) $(FLAGS) -x cu -Xcompiler -fPIC -c $< -o $@

$(OBJ)/trace_main.o: $(HERE)ref_plugin_main.cu | $(OBJ)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/libref_host.so: $(HOST_OBJS) $(OBJ)/shim.o
	$(NVCC) $(ARCH) -shared -o $@ $^

$(OUT)/gpe_ref: $(OBJ)/main.o $(SRC_OBJS) $(HAM_OBJS)
	$(NVCC) $(ARCH) -o $@ $^ -lcufft

$(OUT)/gpe_ref_trace: $(OBJ)/trace_main.o $(SRC_OBJS) $(HAM_OBJS)
	$(NVCC) $(ARCH) -o $@ $^ -lcufft

clean:
	rm -rf $(OUT)

.PHONY: all host clean
