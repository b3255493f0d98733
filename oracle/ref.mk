# Compiles rypath's own host-compilable sources, where they lie in a rypath checkout, into
# oracle/_ref/: libref.so, the pin for the oracle's restatement; libref_image.so, rypath's
# image shader headers and host image sources (with the PNG / JPEG decoders they link);
# libref_demo.so, the demo model; libref_shapes.so, the bilinear patch and analytic shape
# shaders; and
# roulette_known_answers,
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

IMAGE_SRC := $(HERE)ref_image_probe.cpp $(HERE)ref_image_host.cpp $(REF)/src/image_texture.cpp \
	$(REF)/src/environment_sampling.cpp $(REF)/src/rgb_spectrum.cpp $(REF)/src/pbrt_spectra.cpp \
	$(REF)/src/light_sampling.cpp $(REF)/src/png_allocator.cpp $(REF)/third_party/lodepng/lodepng.cpp \
	$(REF)/src/texture_footprint.cpp $(REF)/src/geometry.cpp $(REF)/src/bilinear.cpp \
	$(REF)/third_party/stb/jpeg.cpp
IMAGE_FLAGS := $(FLAGS) -I$(REF)/third_party/stb -I$(REF)/third_party/lodepng -I$(REF)/third_party/pbrt \
	-DRYPATH_SRGB_BIN='"$(REF)/third_party/pbrt/srgb.bin"'

# the demo model: src/render.cpp with what it links, rypath's CPU demo reference
# (tests/render_reference.cpp) and the CIE table header rypath's CMake generates from
# third_party/cie (cmake/CieData.cmake); generated here the same way into the build folder
DEMO_SRC := $(HERE)ref_demo_probe.cpp $(HERE)ref_image_host.cpp $(REF)/src/render.cpp $(REF)/tests/render_reference.cpp \
	$(REF)/src/image_texture.cpp $(REF)/src/environment_sampling.cpp $(REF)/src/rgb_spectrum.cpp \
	$(REF)/src/pbrt_spectra.cpp $(REF)/src/light_sampling.cpp $(REF)/src/png_allocator.cpp \
	$(REF)/third_party/lodepng/lodepng.cpp $(REF)/src/texture_footprint.cpp $(REF)/src/geometry.cpp \
	$(REF)/src/bilinear.cpp $(REF)/third_party/stb/jpeg.cpp $(REF)/src/gaussian_filter.cpp \
	$(REF)/src/texture_graph.cpp $(REF)/src/bsdf_table.cpp $(REF)/src/sampling.cpp $(REF)/src/area_power.cpp \
	$(REF)/src/packet_film.cpp

all: $(OUT)/libref.so $(OUT)/libref_image.so $(OUT)/libref_demo.so $(OUT)/libref_shapes.so $(OUT)/roulette_known_answers

# the procedural primitive shaders (shaders/bilinear.h, shaders/analytic.h)
$(OUT)/libref_shapes.so: $(HERE)ref_shape_probe.cpp $(REF)/shaders/bilinear.h $(REF)/shaders/analytic.h $(HERE)ref_shim/metal_stdlib
	mkdir -p $(OUT)
	$(CXX) $(FLAGS) -Wl,--no-undefined -o $@ $(HERE)ref_shape_probe.cpp

$(OUT)/gen/cie_xyz_data.hpp: $(REF)/third_party/cie/CIE_xyz_1931_2deg.csv
	mkdir -p $(OUT)/gen
	( echo '#pragma once'; echo '#include <array>'; echo 'namespace rypath::detail {'; \
	  echo 'inline constexpr std::array<std::array<double, 3>, 471> cie_xyz{{'; \
	  sed -E 's/^[0-9]+,(.*)$$/    {\1},/' $<; echo '}};'; echo '}' ) > $@

$(OUT)/libref_demo.so: $(DEMO_SRC) $(OUT)/gen/cie_xyz_data.hpp
	mkdir -p $(OUT)
	$(CXX) $(BASE) -shared -I$(OUT)/gen -I$(REF)/src -I$(REF)/tests -I$(REF)/shaders -I$(REF)/third_party/pbrt \
		-I$(REF)/third_party/stb -I$(REF)/third_party/lodepng -DRYPATH_SRGB_BIN='"$(REF)/third_party/pbrt/srgb.bin"' \
		-Wl,--no-undefined -o $@ $(DEMO_SRC)

$(OUT)/libref.so: $(SRC) $(HERE)ref_shim/metal_stdlib
	mkdir -p $(OUT)
	$(CXX) $(FLAGS) -o $@ $(SRC)

# Metal's constant address space is read-only, which C++ spells const: the image probe maps
# `constant` to `const`, and this rule writes a copy of shaders/image_lighting.h into the
# build folder with the one spelling that mapping would double (`const constant` -> `const`).
$(OUT)/gen/image_lighting.h: $(REF)/shaders/image_lighting.h
	mkdir -p $(OUT)/gen
	sed 's/const constant /const /g' $< > $@

$(OUT)/libref_image.so: $(IMAGE_SRC) $(HERE)ref_shim/metal_stdlib $(OUT)/gen/image_lighting.h
	mkdir -p $(OUT)
	$(CXX) -I$(OUT)/gen $(IMAGE_FLAGS) -Wl,--no-undefined -o $@ $(IMAGE_SRC)

$(OUT)/roulette_known_answers: $(REF)/tests/packet_roulette_tests.cpp $(HERE)roulette_as_ref/packet_roulette_shared.h $(HERE)oracle_math.hpp
	mkdir -p $(OUT)
	$(CXX) $(BASE) -I$(HERE)roulette_as_ref -I$(HERE) -I$(REF)/src -o $@ $<

.PHONY: all
