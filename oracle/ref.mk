# Compiles the reference's own kernels (from the reference sources in place)
# plus oracle/ref_harness.cu, oracle/ref_grid_harness.cu and
# oracle/ref_rigid_harness.cu into
# oracle/_ref/librefkernels.so, and the reference's host-side barostat code
# (FixNoseHoover.cu's MTK propagator, FixPressureBerendsen.cu's step) with
# oracle/ref_nh_harness.cu and oracle/ref_berendsen_harness.cu into
# oracle/_ref/librefbarostat.so, which needs no GPU; and the reference's P3M
# splitting-parameter solve (FixChargeEwald.cu) with oracle/ref_ewald_harness.cu
# into oracle/_ref/librefewald.so (host code, but the fix's device arrays
# initialise the CUDA runtime, so it runs where a GPU is).  Test infrastructure only; run where the
# reference is mounted, the .so travels to the GPU box.  Flags follow the
# reference's CMakeLists.txt:53.
# The reference source tree: $(MDX_REFERENCE_SRC) when set, else the default
# below; the target is skipped (with a note) when the tree is absent.
REF ?= $(or $(MDX_REFERENCE_SRC),/root/reference/src)
NVCC ?= /usr/local/cuda/bin/nvcc
CUDA_INC ?= $(dir $(NVCC))../targets/x86_64-linux/include
INC = -I ref_shim -I $(REF) -I $(REF)/Evaluators -I $(REF)/GPUArrays -I $(REF)/Fixes -I $(REF)/DataStorageUser
FLAGS = -gencode arch=compute_100a,code=sm_100a -std=c++14 -Xcompiler -fPIC --use_fast_math --prec-div=true \
        --prec-sqrt=true -O3 -w
# GridGPU.cu and FixRigid.cu include State.h, Fix.h, Bond.h, ... with quotes
# from their own directories; the split include path (-I-) stops those
# directories from being searched first, so that the stand-ins in
# ref_shim_grid/ and ref_shim_rigid/ are found instead.  Quote includes of
# CUDA's own headers and of nvcc's temporary files then need their
# directories before the split.
GRID_TMP = _ref/tmp
REF_DIRS = -I $(REF) -I $(REF)/Evaluators -I $(REF)/GPUArrays -I $(REF)/Fixes -I $(REF)/DataStorageUser \
           -I $(REF)/BondedForcers
GRID_INC = -I ref_shim_grid -I $(CUDA_INC)/crt -I $(CUDA_INC) -I $(GRID_TMP) -I- -I ref_shim_grid $(REF_DIRS)
RIGID_INC = -I ref_shim_rigid -I $(CUDA_INC)/crt -I $(CUDA_INC) -I $(GRID_TMP) -I- -I ref_shim_rigid $(REF_DIRS)
EWALD_INC = -I ref_shim_ewald -I $(CUDA_INC)/crt -I $(CUDA_INC) -I $(GRID_TMP) -I- -I ref_shim_ewald $(REF_DIRS)
NH_INC = -I ref_shim_nh -I $(CUDA_INC)/crt -I $(CUDA_INC) -I $(GRID_TMP) -I- -I ref_shim_nh $(REF_DIRS)

all: _ref/librefkernels.so _ref/librefbarostat.so _ref/librefewald.so

ifeq ($(wildcard $(REF)/Evaluators/PairEvaluateIso.h),)
_ref/librefkernels.so _ref/librefbarostat.so _ref/librefewald.so:
	@echo "reference sources not found under $(REF): oracle/_ref not built"
else
_ref/librefkernels.so: _ref/ref_harness.o _ref/ref_grid_harness.o _ref/ref_rigid_harness.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -o $@ $^

_ref/ref_harness.o: ref_harness.cu
	@mkdir -p _ref
	$(NVCC) $(FLAGS) $(INC) -c -o $@ ref_harness.cu

_ref/ref_grid_harness.o: ref_grid_harness.cu $(wildcard ref_shim_grid/*.h ref_shim_grid/boost/*.hpp)
	@mkdir -p _ref $(GRID_TMP)
	TMPDIR=$(abspath $(GRID_TMP)) $(NVCC) $(FLAGS) $(GRID_INC) -c -o $@ ref_grid_harness.cu

_ref/ref_rigid_harness.o: ref_rigid_harness.cu $(wildcard ref_shim_rigid/*.h ref_shim_rigid/boost/*.hpp)
	@mkdir -p _ref $(GRID_TMP)
	TMPDIR=$(abspath $(GRID_TMP)) $(NVCC) $(FLAGS) $(RIGID_INC) -c -o $@ ref_rigid_harness.cu

_ref/librefbarostat.so: _ref/ref_nh_harness.o _ref/ref_berendsen_harness.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -o $@ $^

_ref/ref_nh_harness.o: ref_nh_harness.cu $(wildcard ref_shim_nh/*.h ref_shim_nh/boost/*.hpp ref_shim_nh/boost/python/*)
	@mkdir -p _ref $(GRID_TMP)
	TMPDIR=$(abspath $(GRID_TMP)) $(NVCC) $(FLAGS) $(NH_INC) -c -o $@ ref_nh_harness.cu

_ref/ref_berendsen_harness.o: ref_berendsen_harness.cu $(wildcard ref_shim_nh/*.h ref_shim_nh/boost/*.hpp ref_shim_nh/boost/python/*)
	@mkdir -p _ref $(GRID_TMP)
	TMPDIR=$(abspath $(GRID_TMP)) $(NVCC) $(FLAGS) $(NH_INC) -c -o $@ ref_berendsen_harness.cu

_ref/librefewald.so: _ref/ref_ewald_harness.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -o $@ $^ -lcufft

_ref/ref_ewald_harness.o: ref_ewald_harness.cu $(wildcard ref_shim_ewald/*.h ref_shim_ewald/boost/*.hpp ref_shim_ewald/boost/python/*)
	@mkdir -p _ref $(GRID_TMP)
	TMPDIR=$(abspath $(GRID_TMP)) $(NVCC) $(FLAGS) $(EWALD_INC) -c -o $@ ref_ewald_harness.cu
endif

clean:
	rm -rf _ref

.PHONY: all clean
