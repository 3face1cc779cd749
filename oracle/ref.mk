# Test infrastructure: builds the reference implementation, from its sources
# where they lie, into oracle/_ref/ (git-ignored).  Used only as a checker by
# tests/ and by bench.py's CPU-baseline leg; the product never links it.
#
#   make -f oracle/ref.mk [REF=<reference tree>]        (from the repo root)
#   make -s -f oracle/ref.mk refdir                      (prints the tree used)
#
# The reference tree is REF, else $ASDM_REFERENCE_DIR, else the default below;
# this recipe is the one place that names it (tests and the build entry point
# ask it with `refdir`).
#
# No reference build system is run: GLPK 4.55's C sources and the reference's
# C++ sources are compiled directly with the flags below (GLPK's shipped
# object files and archives are neither read nor linked; everything is
# rebuilt from .c/.cpp).  The reference's compile-time modes
# (config/config.h:38-40) are passed with -D, which config.h leaves alone
# because its own #defines of them are commented out.
REF      ?= $(or $(ASDM_REFERENCE_DIR),/root/reference)
OUT      ?= oracle/_ref
CXX      ?= g++
CC       ?= gcc
JOBS     ?= 8

GLPK_SRC := $(REF)/utility/td/glpk-4.55/src
GLPK_DIRS := $(GLPK_SRC) $(addprefix $(GLPK_SRC)/,amd bflib cglib colamd env minisat misc proxy zlib)
GLPK_C   := $(foreach d,$(GLPK_DIRS),$(wildcard $(d)/*.c))
GLPK_INC := $(addprefix -I,$(GLPK_DIRS))

# Reference C++ sources of the matching path (entry points main.cpp and
# executable/prepare.cpp are replaced by oracle/ref_harness.cpp).
REF_CPP  := $(REF)/relation/candidate_space.cpp $(REF)/relation/graph.cpp \
            $(REF)/relation/relation.cpp $(REF)/relation/dynamic_array.cpp \
            $(REF)/plan/decomposition.cpp $(REF)/plan/estimator.cpp \
            $(REF)/plan/optimizer.cpp $(REF)/plan/subset_structure.cpp \
            $(REF)/matching/join.cpp $(REF)/matching/adaptive.cpp \
            $(REF)/utility/command_parser.cpp $(REF)/utility/utils.cpp \
            $(REF)/utility/command.cpp $(REF)/utility/compute_set_intersection.cpp \
            $(REF)/utility/td/dataloader.cpp $(REF)/utility/td/hypergraph.cpp \
            $(REF)/utility/td/preprocessing.cpp $(REF)/utility/td/td.cpp \
            $(REF)/utility/td/twbound.cpp $(REF)/utility/td/SCsolver.cpp
REF_INC  := -I$(REF)/config -I$(REF)/utility -I$(REF)/relation -I$(REF)/plan \
            -I$(REF)/matching -I$(REF)/utility/td -I$(GLPK_SRC)
# -include cstdint: utility/td/hypergraph.h uses uint64_t without <cstdint>
# (GCC 13 no longer pulls it in transitively).
CXXFLAGS_REF := -std=c++17 -O3 -march=x86-64-v3 -include cstdint -w $(REF_INC)

GLPK_OBJ := $(patsubst $(REF)/%.c,$(OUT)/obj/%.o,$(GLPK_C))

VARIANTS := ref_count ref_local ref_embed
DEF_ref_count := -DALL_LEVEL
DEF_ref_local := -DALL_LEVEL -DLOCAL_COUNT
DEF_ref_embed := -DALL_LEVEL -DLOCAL_COUNT -DCOLLECT_RESULT

all: $(addprefix $(OUT)/,$(VARIANTS))

$(OUT)/obj/%.o: $(REF)/%.c
	@mkdir -p $(dir $@)
	$(CC) -O2 -w $(GLPK_INC) -c $< -o $@

$(OUT)/libglpk_src.a: $(GLPK_OBJ)
	ar rcs $@ $^

define VARIANT_RULE
$(OUT)/$(1): oracle/ref_harness.cpp $(REF_CPP) $(OUT)/libglpk_src.a
	@mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS_REF) $(DEF_$(1)) oracle/ref_harness.cpp $(REF_CPP) $(OUT)/libglpk_src.a -lpthread -lm -o $$@
endef
$(foreach v,$(VARIANTS),$(eval $(call VARIANT_RULE,$(v))))

refdir:
	@echo $(REF)

clean:
	rm -rf $(OUT)

.PHONY: all clean refdir
