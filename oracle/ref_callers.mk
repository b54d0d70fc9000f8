# Builds the reference's own C test programs and Python wrappers, unmodified,
# from where they lie in the reference tree, against this repository's
# library: the evidence that libfteik_shared.so is a drop-in for their calls.
# Test infrastructure only; outputs go to oracle/_ref/ (git-ignored).
#
#   testing/loctest.c              -> _ref/loctest       (locator known answer)
#   performanceTests/convergence.c -> _ref/convergence   (2D first-order convergence)
#   python/fteik3d.py, fteik2d.py  -> _ref/python/*.bytecode (byte-compiled, loaded sourceless)
#
# The C programs include "fteik/fteik_fortran.h", found in ../include; they
# link ../fteik_b200/lib/libfteik_shared.so through an $ORIGIN-relative rpath,
# so the binaries run wherever this repository is copied.
REF ?= /root/reference
ROOT := $(abspath ..)
OUT := _ref
CC := gcc
PY ?= python3
CFLAGS := -O2 -std=gnu11 -I$(ROOT)/include
LDFLAGS := -L$(ROOT)/fteik_b200/lib -lfteik_shared -Wl,-rpath,'$$ORIGIN/../../fteik_b200/lib' -lm

ifeq ($(wildcard $(REF)/testing/loctest.c),)
all:
	@echo "ref_callers.mk: no reference tree at $(REF); the callers are not built"
else
all: $(OUT)/loctest $(OUT)/convergence $(OUT)/python/fteik3d.bytecode $(OUT)/python/fteik2d.bytecode
endif

$(OUT):
	mkdir -p $(OUT)/python

$(OUT)/loctest: $(REF)/testing/loctest.c $(ROOT)/include/fteik_b200.h | $(OUT)
	$(CC) $(CFLAGS) -o $@ $< $(LDFLAGS)

$(OUT)/convergence: $(REF)/performanceTests/convergence.c $(ROOT)/include/fteik_b200.h | $(OUT)
	$(CC) $(CFLAGS) -o $@ $< $(LDFLAGS)

$(OUT)/python/%.bytecode: $(REF)/python/%.py | $(OUT)
	$(PY) -c "import py_compile, sys; py_compile.compile(sys.argv[1], cfile=sys.argv[2], doraise=True)" $< $@

.PHONY: all
