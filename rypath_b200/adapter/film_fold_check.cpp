// SPDX-License-Identifier: GPL-3.0-only
// Checks film_fold against rypath's FilmPixel layout (src/render.hpp:317-339): a Film unfolded
// into device rows and folded back is the same Film; every field lands where the device film
// keeps it; a Film with splat sums (which the hero transport never produces) is refused.
// Built by rypath_b200/adapter/Makefile; exits 0 when every check holds.
#include "film_fold.hpp"

#include <cstdio>
#include <vector>

int main() {
    using namespace rypath;
    Film film;
    film.width = 7;
    film.height = 5;
    film.pixels.resize(35);
    double v = 1.0;
    for (FilmPixel &p : film.pixels) {
        for (int c = 0; c < 3; ++c) {
            p.sum[c] = v *= 1.37;
            p.correction[c] = -v * 1e-17;
            p.compatibility_sum[c] = v * 0.5;
            p.compatibility_correction[c] = v * 3e-18;
        }
        p.weight_sum = v * 0.25;
        p.weight_correction = -v * 1e-19;
        p.count = std::uint64_t(v) % 1000 + 1;
    }
    std::vector<rp_film_pixel> rows(film.pixels.size());
    if (!cuda_backend::unfold_film(film, rows).empty())
        return std::puts("unfold refused a splat-free Film"), 1;
    for (std::size_t i = 0; i < rows.size(); ++i) {
        const FilmPixel &p = film.pixels[i];
        const rp_film_pixel &r = rows[i];
        for (int c = 0; c < 3; ++c)
            if (r.sum[c] != p.sum[c] || r.correction[c] != p.correction[c] ||
                r.compatibility_sum[c] != p.compatibility_sum[c] ||
                r.compatibility_correction[c] != p.compatibility_correction[c] || r.square[c] != 0)
                return std::puts("a colour plane landed in the wrong device field"), 1;
        if (r.weight_sum != p.weight_sum || r.weight_correction != p.weight_correction || r.count != p.count)
            return std::puts("weights or counts landed in the wrong device field"), 1;
    }
    Film back = film;
    for (FilmPixel &p : back.pixels)
        p = {};
    if (!cuda_backend::fold_film(rows, back).empty() || !(back == film))
        return std::puts("fold(unfold(film)) differs from the film"), 1;
    Film splatted = film;
    splatted.pixels[3].splat_sum[1] = 1;
    if (cuda_backend::unfold_film(splatted, rows).empty())
        return std::puts("a Film with splat sums was accepted"), 1;
    std::vector<rp_film_pixel> short_rows(3);
    if (cuda_backend::unfold_film(film, short_rows).empty() || cuda_backend::fold_film(short_rows, back).empty())
        return std::puts("a size mismatch was accepted"), 1;
    std::puts("film fold ok");
    return 0;
}
