// SPDX-License-Identifier: GPL-3.0-only
// What the B200 backend adds to rypath's GPU backend boundary (src/metal_render.hpp): whole
// batches of a progressive render into rypath's Film, reduced on the device, for a driver that
// wants the committed Film without reading every lane back.  build_metal_renderer and
// MetalRenderScene::sample themselves keep the declarations of src/metal_render.hpp.
#pragma once
#include "render.hpp"

#include <cstdint>
#include <memory>
#include <string>

struct rp_scene;

namespace rypath::cuda_backend {

class FilmRenderer {
  public:
    // The device scene of `scene` on device 0; nullptr with `diag` set on failure.
    static std::unique_ptr<FilmRenderer> build(const RenderScene &scene, std::string &diag);
    ~FilmRenderer();
    FilmRenderer(const FilmRenderer &) = delete;
    FilmRenderer &operator=(const FilmRenderer &) = delete;

    // Samples [sample_begin, sample_begin + count) of every pixel, settings.batch_size absolute
    // samples per batch, onto `film`'s committed sums (a fresh render when sample_begin is 0; a
    // resumed one, as after a checkpoint restore, uploads `film` first).  Returns the
    // diagnostic of a failed batch, which leaves `film` as committed before that batch
    // (src/render_driver.cpp:201-214); empty on success.
    std::string render(const RenderSettings &settings, std::uint64_t sample_begin, std::uint64_t count, Film &film);

  private:
    explicit FilmRenderer(rp_scene *scene) : scene_(scene) {}
    rp_scene *scene_;
};

} // namespace rypath::cuda_backend
