# Builds the reference CellSim3D CUDA kernels, unmodified, from the
# reference sources where they lie, together with ref_harness.cu (the
# reference's timestep driven from an input file) into oracle/_ref/cs3d_ref.
# Test and baseline infrastructure only; the outputs stay out of git.
#
#   make -f oracle/ref.mk [REF=/path/to/CellSim3D]
#
# REF defaults to $CELLSIM3D_REF, else to a CellSim3D checkout named
# `reference` beside this repository.
HERE0 := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
REF ?= $(if $(CELLSIM3D_REF),$(CELLSIM3D_REF),$(abspath $(HERE0)../../reference))
NVCC ?= nvcc
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref
ARCH := -gencode arch=compute_100a,code=sm_100a
# the reference's own flags (makefile: -O3 -dc -D_FORCE_INLINES -I inc),
# with the architecture raised to sm_100a
FLAGS := $(ARCH) -O3 -rdc=true -D_FORCE_INLINES -I$(REF)/inc -I$(REF)/src -w
KERNELS := centermass postscriptinit PressureKernels propagatebound propagate volume
OBJS := $(patsubst %,$(OUT)/%.o,$(KERNELS))

all: $(OUT)/cs3d_ref

$(OUT):
	mkdir -p $@

$(OUT)/%.o: $(REF)/src/%.cu | $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/ref_harness.o: $(HERE)ref_harness.cu $(HERE)../include/cs3d.h | $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/cs3d_ref: $(OBJS) $(OUT)/ref_harness.o
	$(NVCC) $(ARCH) -rdc=true -o $@ $^ -lcurand

.PHONY: all
