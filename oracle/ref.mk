# Compiles rypath's own host-compilable sources, where they lie in a rypath checkout, into
# oracle/_ref/: libref.so, the pin for the oracle's restatement, and roulette_known_answers,
# rypath's own roulette test program built against the oracle's restatement of the roulette
# header (oracle/roulette_as_ref).  Test infrastructure only; not rypath's build system.
# Usage: make -f oracle/ref.mk REF=/path/to/rypath
ifeq ($(REF),)
$(error REF must name a rypath checkout: make -f oracle/ref.mk REF=/path/to/rypath)
endif
CXX ?= g++
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT := $(HERE)_ref
BASE := -O2 -std=c++20 -fPIC -ffp-contract=off -fno-fast-math -w
FLAGS := $(BASE) -shared -I$(REF)/src -I$(REF)/shaders -I$(HERE)ref_shim
SRC := $(HERE)ref_probe.cpp $(HERE)ref_hero_probe.cpp $(REF)/src/light_sampling.cpp $(REF)/src/packet_film.cpp

all: $(OUT)/libref.so $(OUT)/roulette_known_answers

$(OUT)/libref.so: $(SRC) $(HERE)ref_shim/metal_stdlib
	mkdir -p $(OUT)
	$(CXX) $(FLAGS) -o $@ $(SRC)

$(OUT)/roulette_known_answers: $(REF)/tests/packet_roulette_tests.cpp $(HERE)roulette_as_ref/packet_roulette_shared.h $(HERE)oracle_math.hpp
	mkdir -p $(OUT)
	$(CXX) $(BASE) -I$(HERE)roulette_as_ref -I$(HERE) -I$(REF)/src -o $@ $<

.PHONY: all
