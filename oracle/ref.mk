# Compiles the reference's own headers (sparxastronomy/fasttree src/*.hpp, read in place)
# against the host SYCL/oneDPL stand-ins in sycl_shim/, one shared object per compile-time
# configuration, into oracle/_ref/.  Test infrastructure only (the checker).
#
#   make -C oracle -f ref.mk REF_SRC=<reference checkout>/src
#
# The Morton configuration does not compile as shipped (see sycl_shim/morton_prelude.hpp);
# its builds force-include that prelude, which declares the four missing names.
ifeq ($(REF_SRC),)
REF_SRC  := $(FASTTREE_REF_SRC)
endif
ifeq ($(REF_SRC),)
$(error set REF_SRC (or FASTTREE_REF_SRC) to the reference's src/ directory)
endif
CXX      := $(if $(wildcard /usr/bin/g++),/usr/bin/g++,g++)
CXXFLAGS ?= -O2 -std=c++20 -fopenmp -ffp-contract=off -fPIC -shared -w -fno-strict-aliasing
INC      := -Isycl_shim -I$(REF_SRC)
OUT      := _ref

MORTON := -DSFC_TYPE_MORTON -include sycl_shim/morton_prelude.hpp
PH     := -DSFC_TYPE_PEANO_HILBERT
INT32  := -DFASTTREE_INTEGER_COORDS -DPOSITIONS_IN_32BIT
INT64  := -DFASTTREE_INTEGER_COORDS -DPOSITIONS_IN_64BIT

CONFIGS := morton_f32 morton_f64 ph_f32 ph_f64 ph_u32 ph_u32_per ph_u64 ph_u64_per morton_f64_orig ph_u64_per_orig

flags_morton_f32      := $(MORTON)
flags_morton_f64      := $(MORTON) -DCOORDS_TYPE_DOUBLE
flags_ph_f32          := $(PH)
flags_ph_f64          := $(PH) -DCOORDS_TYPE_DOUBLE
flags_ph_u32          := $(PH) $(INT32)
flags_ph_u32_per      := $(PH) $(INT32) -DPERIODIC_BC
flags_ph_u64          := $(PH) $(INT64)
flags_ph_u64_per      := $(PH) $(INT64) -DPERIODIC_BC
flags_morton_f64_orig := $(MORTON) -DCOORDS_TYPE_DOUBLE -DRETURN_ORIG_INDICES
flags_ph_u64_per_orig := $(PH) $(INT64) -DPERIODIC_BC -DRETURN_ORIG_INDICES

LIBS := $(foreach c,$(CONFIGS),$(OUT)/libftref_$(c).so)
DEPS := ref_driver.cpp $(wildcard sycl_shim/sycl/*.hpp) $(wildcard sycl_shim/oneapi/dpl/*) \
        $(wildcard $(REF_SRC)/*.hpp)

all: $(LIBS)

$(OUT)/libftref_%.so: $(DEPS)
	@mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) $(INC) $(flags_$*) -o $@ ref_driver.cpp

clean:
	rm -rf $(OUT)

.PHONY: all clean
