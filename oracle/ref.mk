# Compiles the reference's own header kernels (from the reference sources in
# place) plus oracle/ref_harness.cu into oracle/_ref/librefkernels.so.
# Test infrastructure only; run where the reference is mounted, the .so
# travels to the GPU box.  Flags follow the reference's CMakeLists.txt:53.
# The reference source tree: $(MDX_REFERENCE_SRC) when set, else the default
# below; the target is skipped (with a note) when the tree is absent.
REF ?= $(or $(MDX_REFERENCE_SRC),/root/reference/src)
NVCC ?= /usr/local/cuda/bin/nvcc
INC = -I ref_shim -I $(REF) -I $(REF)/Evaluators -I $(REF)/GPUArrays -I $(REF)/Fixes -I $(REF)/DataStorageUser
FLAGS = -gencode arch=compute_100a,code=sm_100a -std=c++14 -Xcompiler -fPIC --use_fast_math --prec-div=true \
        --prec-sqrt=true -O3 -w

ifeq ($(wildcard $(REF)/Evaluators/PairEvaluateIso.h),)
_ref/librefkernels.so:
	@echo "reference sources not found under $(REF): oracle/_ref not built"
else
_ref/librefkernels.so: ref_harness.cu
	@mkdir -p _ref
	$(NVCC) $(FLAGS) $(INC) -shared -o $@ ref_harness.cu
endif

clean:
	rm -rf _ref

.PHONY: clean
