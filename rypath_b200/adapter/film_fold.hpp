// SPDX-License-Identifier: GPL-3.0-only
// Conversion between the B200 backend's device film rows (rp_film_pixel, include/rypath_cuda.h)
// and rypath's committed Film (FilmPixel, src/render.hpp:317-339).  Both hold the same FP64
// Neumaier sums of PacketFilmBatch (src/packet_film.cpp:198-265), so the conversion copies
// words and loses nothing: a committed Film uploaded, rendered onto and folded back equals the
// host reduction of the same lanes bit for bit.  The hero path splats nothing, so the splat
// planes stay zero; the device film's second moments have no FilmPixel field.
#pragma once
#include "render.hpp"
#include <rypath_cuda.h>

#include <span>
#include <string>

namespace rypath::cuda_backend {

// Film pixels -> device rows (second moments zero: a checkpointed Film does not store them).
// Returns a diagnostic for a Film with splat sums, which no hero render produces.
std::string unfold_film(const Film &film, std::span<rp_film_pixel> rows);
// Device rows -> Film pixels (the Film's size and settings are kept).
std::string fold_film(std::span<const rp_film_pixel> rows, Film &film);

} // namespace rypath::cuda_backend
