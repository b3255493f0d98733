// SPDX-License-Identifier: GPL-3.0-only
#include "film_fold.hpp"

namespace rypath::cuda_backend {

std::string unfold_film(const Film &film, std::span<rp_film_pixel> rows) {
    if (rows.size() != film.pixels.size())
        return "device film and Film differ in size";
    for (std::size_t i = 0; i < rows.size(); ++i) {
        const FilmPixel &p = film.pixels[i];
        for (int c = 0; c < 3; ++c)
            if (p.splat_sum[c] != 0 || p.splat_correction[c] != 0 || p.compatibility_splat_sum[c] != 0 ||
                p.compatibility_splat_correction[c] != 0)
                return "Film holds splat sums, which the hero transport does not produce";
        rp_film_pixel &r = rows[i];
        r = {};
        for (int c = 0; c < 3; ++c) {
            r.sum[c] = p.sum[c];
            r.correction[c] = p.correction[c];
            r.compatibility_sum[c] = p.compatibility_sum[c];
            r.compatibility_correction[c] = p.compatibility_correction[c];
        }
        r.weight_sum = p.weight_sum;
        r.weight_correction = p.weight_correction;
        r.count = p.count;
    }
    return {};
}

std::string fold_film(std::span<const rp_film_pixel> rows, Film &film) {
    if (rows.size() != film.pixels.size())
        return "device film and Film differ in size";
    for (std::size_t i = 0; i < rows.size(); ++i) {
        const rp_film_pixel &r = rows[i];
        FilmPixel &p = film.pixels[i];
        p = {};
        for (int c = 0; c < 3; ++c) {
            p.sum[c] = r.sum[c];
            p.correction[c] = r.correction[c];
            p.compatibility_sum[c] = r.compatibility_sum[c];
            p.compatibility_correction[c] = r.compatibility_correction[c];
        }
        p.weight_sum = r.weight_sum;
        p.weight_correction = r.weight_correction;
        p.count = r.count;
    }
    return {};
}

} // namespace rypath::cuda_backend
