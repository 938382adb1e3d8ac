// Datasets: camera bounds and cameras (engine/src/dataset.cpp:60-83, 226-250) and
// synthetic orbit captures rendered through libgs_cuda.
#include "gs/dataset.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <stdexcept>

#include "frame.h"
#include "gs_cuda.h"

namespace gs {

size_t Dataset::train_count() const {
  return size_t(std::count_if(frames.begin(), frames.end(), [](const DatasetFrame& f) { return !f.holdout; }));
}

size_t Dataset::holdout_count() const { return frames.size() - train_count(); }

void compute_camera_bounds(Dataset& ds) {
  if (ds.frames.empty()) return;
  double sum[3] = {0, 0, 0};
  for (const DatasetFrame& f : ds.frames)
    for (int k = 0; k < 3; ++k) sum[k] += f.c2w[k * 4 + 3];
  for (int k = 0; k < 3; ++k) ds.camera_center[k] = float(sum[k] / double(ds.frames.size()));
  float max_dist = 0.0f;
  for (const DatasetFrame& f : ds.frames) {
    float d2 = 0.0f;
    for (int k = 0; k < 3; ++k) {
      const float d = f.c2w[k * 4 + 3] - ds.camera_center[k];
      d2 += d * d;
    }
    max_dist = std::max(max_dist, std::sqrt(d2));
  }
  ds.camera_extent = std::max(1.1f * max_dist, 1e-3f);
}

Camera dataset_camera(const Dataset& ds, const DatasetFrame& f) {
  if (f.width != 0) return camera_from_c2w_gl(f.c2w, f.fx, f.fy, f.cx, f.cy, f.width, f.height);
  return camera_from_c2w_gl(f.c2w, ds.fx, ds.fy, ds.cx, ds.cy, ds.width, ds.height);
}

Dataset make_orbit_capture(const SplatScene& truth, const OrbitCaptureOptions& o) {
  if (o.cameras == 0 || o.resolutions.empty()) throw std::runtime_error("make_orbit_capture: no cameras");
  Dataset ds;
  ds.name = "synthetic orbit";
  const Resolution& first = o.resolutions.front();
  ds.width = first.width;
  ds.height = first.height;
  ds.fx = ds.fy = first.focal;
  ds.cx = 0.5f * float(first.width);
  ds.cy = 0.5f * float(first.height);
  std::mt19937_64 rng(o.seed);
  std::vector<double> weights;
  for (const Resolution& r : o.resolutions) weights.push_back(r.probability);
  std::discrete_distribution<size_t> pick(weights.begin(), weights.end());
  const bool mixed = o.resolutions.size() > 1;
  ds.frames.resize(o.cameras);
  for (uint32_t i = 0; i < o.cameras; ++i) {
    DatasetFrame& f = ds.frames[i];
    f.name = "orbit_" + std::to_string(i);
    const float a = 2.0f * 3.14159265358979f * float(i) / float(o.cameras);
    const float eye[3] = {o.radius * std::sin(a), o.height, o.radius * std::cos(a)};
    const float target[3] = {0.0f, 0.0f, 0.0f};
    look_at_c2w_gl(eye, target, f.c2w);
    f.holdout = o.holdout_every > 0 && i % o.holdout_every == 0;
    const Resolution& r = o.resolutions[mixed ? pick(rng) : 0];
    if (mixed) {
      f.width = r.width;
      f.height = r.height;
      f.fx = f.fy = r.focal;
      f.cx = 0.5f * float(r.width);
      f.cy = 0.5f * float(r.height);
    }
  }
  compute_camera_bounds(ds);

  // Targets: the truth rendered over black, alpha 255 (no masks).
  gs_context* ctx = nullptr;
  detail::check_status(gs_create(o.device, &ctx), "make_orbit_capture");
  try {
    const uint32_t stride = uint32_t(sh_rest_coeffs(truth.sh_degree) * 3);
    std::vector<float> p, sh;
    detail::pack_params(truth, truth.sh_degree, stride, p, sh);
    detail::check_status(gs_model_init(ctx, std::max(truth.count, 1u), stride, p.data(), stride ? sh.data() : nullptr,
                                       truth.count),
                         "make_orbit_capture: gs_model_init");
    const float black[3] = {0.0f, 0.0f, 0.0f};
    for (DatasetFrame& f : ds.frames) {
      const Camera cam = dataset_camera(ds, f);
      gs_frame_data fd;
      detail::frame_geometry(fd, cam, truth.count, stride, truth.sh_degree, 0u, black);
      f.rgba.assign(size_t(cam.width) * cam.height * 4, 0);
      detail::check_status(gs_render(ctx, &fd, f.rgba.data()), "make_orbit_capture: gs_render");
      for (size_t px = 3; px < f.rgba.size(); px += 4) f.rgba[px] = 255;
    }
  } catch (...) {
    gs_destroy(ctx);
    throw;
  }
  gs_destroy(ctx);
  return ds;
}

}  // namespace gs
