# Compiles rypath's own host-compilable sources, where they lie in a rypath checkout, into
# oracle/_ref/libref.so -- the pin for the oracle's restatement.  Test infrastructure
# only; not rypath's build system.  Usage: make -f oracle/ref.mk REF=/path/to/rypath
REF ?= /root/reference
CXX ?= g++
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref
FLAGS := -O2 -std=c++20 -fPIC -ffp-contract=off -fno-fast-math -w -shared \
	-I$(REF)/src -I$(REF)/shaders -I$(HERE)ref_shim
SRC := $(HERE)ref_probe.cpp $(REF)/src/light_sampling.cpp $(REF)/src/packet_film.cpp

$(OUT)/libref.so: $(SRC) $(HERE)ref_shim/metal_stdlib
	mkdir -p $(OUT)
	$(CXX) $(FLAGS) -o $@ $(SRC)
