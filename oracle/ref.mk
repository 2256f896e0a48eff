# Builds the reference projector library (wudufan/CTProjector, kernel/projector/cuda)
# from its own sources, for sm_100a, into oracle/_ref/libprojector.so, and its
# TV prior (kernel/prior/cuda/TotalVariation.cu) into oracle/_ref/libprior.so.
#
# This is test infrastructure: the library is the GPU oracle that produces the
# golden fixtures under tests/golden/ and the timed reference arm of bench.py.
# It is never linked into, or called by, the ctprojector_b200 product path.
#
#   make -f oracle/ref.mk [REF=<reference checkout>]   (run from the repo root)
#
# REF defaults to $(CTP_REFERENCE_SRC) or the checkout of this build machine;
# without the sources the recipe does nothing.  The sources are read where
# they lie; nothing is copied into this repository.

REF     ?= $(or $(CTP_REFERENCE_SRC),/root/reference)
SRC_DIR := $(REF)/src/ct_projector/kernel/projector/cuda
PRIOR   := $(REF)/src/ct_projector/kernel/prior/cuda/TotalVariation.cu
OUT     := oracle/_ref
OBJ_DIR := $(OUT)/obj
NVCC    ?= nvcc
ARCH    := -gencode arch=compute_100a,code=sm_100a

SOURCES := $(wildcard $(SRC_DIR)/*.cu)
OBJECTS := $(patsubst $(SRC_DIR)/%.cu,$(OBJ_DIR)/%.o,$(SOURCES))

.PHONY: all clean

ifeq ($(SOURCES),)
all:
	@echo "ref.mk: no reference sources under $(REF); oracle/_ref not built"
else
all: $(OUT)/libprojector.so $(OUT)/libprior.so
endif

$(OUT)/libprojector.so: $(OBJECTS)
	$(NVCC) --shared $(ARCH) $(OBJECTS) -lcufft -o $@

# The reference defines device helpers in one translation unit and calls them
# from another, so it needs relocatable device code (-dc) and a device link.
$(OBJ_DIR)/%.o: $(SRC_DIR)/%.cu | $(OBJ_DIR)
	$(NVCC) -O3 $(ARCH) -I$(SRC_DIR)/.. -dc --compiler-options '-fPIC' -w $< -o $@

# one self-contained translation unit
$(OUT)/libprior.so: $(PRIOR) | $(OBJ_DIR)
	$(NVCC) -O3 $(ARCH) --shared --compiler-options '-fPIC' -w $< -o $@

$(OBJ_DIR):
	mkdir -p $(OBJ_DIR)

clean:
	rm -rf $(OUT)
