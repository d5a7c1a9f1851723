# Builds the unmodified reference PCAone (v0.6.0) CLI from the read-only source tree
# into oracle/_ref/ for use as the parity oracle and the timed CPU baseline.
#
#   make -f oracle/ref.mk REF=<reference source tree> -j8
# (REF defaults to $PCAONE_REF, else /root/reference)
#
# This is our own short recipe (the reference's own build system is not run).
# Sources are compiled where they lie; objects and the binary go to oracle/_ref/ only.
# -march=x86-64-v3 (AVX2+FMA) instead of -march=native so the binary also runs on the
# host CPU of another machine; OpenMP is enabled as in the reference build.

REF      ?= $(if $(PCAONE_REF),$(PCAONE_REF),/root/reference)
OUT      := $(dir $(lastword $(MAKEFILE_LIST)))_ref
OBJ      := $(OUT)/obj
CXX      := /usr/bin/g++
CC       := /usr/bin/gcc
ARCHFLAG ?= -march=x86-64-v3
CXXFLAGS := -O3 -std=c++17 -m64 -DNDEBUG $(ARCHFLAG) -fopenmp -DVERSION=\"0.6.0\" -w
CFLAGS   := -O3 -m64 -DNDEBUG $(ARCHFLAG) -DZSTD_DISABLE_ASM -DZSTD_MULTITHREAD=0 -w
INC      := -I$(REF)/external -I$(REF)/external/zstd/lib -I$(REF)/external/zstd/lib/common

PCA_SRC  := Arnoldi Halko Data Utils Cmd FileBeagle FileCsv FileBgen FilePlink FileBinary \
            FileUSV LD Projection Inbreeding kfunc Main
BGEN_SRC := $(notdir $(basename $(wildcard $(REF)/external/bgen/*.cpp)))
ZSTD_SRC := $(wildcard $(REF)/external/zstd/lib/common/*.c) \
            $(wildcard $(REF)/external/zstd/lib/compress/*.c) \
            $(wildcard $(REF)/external/zstd/lib/decompress/*.c)

PCA_OBJ  := $(addprefix $(OBJ)/pca_,$(addsuffix .o,$(PCA_SRC)))
BGEN_OBJ := $(addprefix $(OBJ)/bgen_,$(addsuffix .o,$(BGEN_SRC)))
ZSTD_OBJ := $(addprefix $(OBJ)/zstd_,$(notdir $(ZSTD_SRC:.c=.o)))

all: $(OUT)/PCAone

$(OUT)/PCAone: $(PCA_OBJ) $(BGEN_OBJ) $(ZSTD_OBJ)
	$(CXX) $(CXXFLAGS) -o $@ $^ -lz -lgomp -lpthread -ldl -lm

$(OBJ)/pca_%.o: $(REF)/src/%.cpp | $(OBJ)
	$(CXX) $(CXXFLAGS) $(INC) -c $< -o $@

$(OBJ)/bgen_%.o: $(REF)/external/bgen/%.cpp | $(OBJ)
	$(CXX) $(CXXFLAGS) -I$(REF)/external/zstd/lib -c $< -o $@

define zstd_rule
$(OBJ)/zstd_$(notdir $(1:.c=.o)): $(1) | $(OBJ)
	$(CC) $(CFLAGS) -I$(REF)/external/zstd/lib -I$(REF)/external/zstd/lib/common -c $$< -o $$@
endef
$(foreach s,$(ZSTD_SRC),$(eval $(call zstd_rule,$(s))))

$(OBJ):
	mkdir -p $@

.PHONY: all

# Dump of the reference's own Omega / permutation draws (pins oracle/rng.cpp).
all: $(OUT)/omega_ref
$(OUT)/omega_ref: $(dir $(lastword $(MAKEFILE_LIST)))ref_omega.cpp | $(OBJ)
	$(CXX) -O2 -std=c++17 -w -I$(REF)/external -I$(REF)/src -I$(REF)/external/zstd/lib -o $@ $<
