# Builds oracle/_ref/libref_kernel.so: the REFERENCE's pair kernel
# (BoostXmatch/Worker.cu) and RA half-width (BoostXmatch/Common.cu), compiled
# unmodified from the read-only reference tree for sm_100a, linked with the
# harness oracle/ref_harness.cu.  Test infrastructure only; needs the
# reference tree, so it is built in the build container and the .so travels.
#   make -f oracle/ref_kernel.mk [REFERENCE=<reference checkout>]
HERE      := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
REFERENCE ?= /root/reference
REF       ?= $(REFERENCE)/BoostXmatch/BoostXmatch
OUT    := $(HERE)_ref
NVCC   ?= nvcc
FLAGS  := -gencode arch=compute_100a,code=sm_100a -O2 -std=c++17 -Xcompiler -fPIC \
          -I$(HERE)refshim -I$(REF) -diag-suppress 177,550,2361,20011,20012,20013,20014 -w

all: $(OUT)/libref_kernel.so

$(OUT)/Worker.o: $(REF)/Worker.cu
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/Common.o: $(REF)/Common.cu
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -x cu -c $< -o $@

$(OUT)/ref_harness.o: $(HERE)ref_harness.cu
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/libref_kernel.so: $(OUT)/Worker.o $(OUT)/Common.o $(OUT)/ref_harness.o
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -o $@ $^

clean:
	rm -rf $(OUT)

.PHONY: all clean
