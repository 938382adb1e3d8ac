// Datasets: camera bounds and cameras (engine/src/dataset.cpp:60-83, 226-250) and
// synthetic orbit captures rendered through libgs_cuda.
#include "gs/dataset.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <unordered_map>

#include "frame.h"
#include "gs_cuda.h"
#include "image_io.h"

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

HeadRegion estimate_head(const Dataset& dataset, const SplatScene& subject) {
  return estimate_head(subject, dataset.world_up);
}

HeadRegion estimate_head(const SplatScene& subject, const float up[3]) {
  HeadRegion head;
  const size_t n = subject.count;
  if (n < 200) return head;
  // Heights along world up; the extent ignores the lowest 1% and the highest 0.5%.
  std::vector<float> h(n);
  for (size_t i = 0; i < n; ++i) {
    const float* p = &subject.positions[i * 3];
    h[i] = up[0] * p[0] + up[1] * p[1] + up[2] * p[2];
  }
  std::vector<float> order(h);
  std::sort(order.begin(), order.end());
  const float bottom = order[n / 100], top = order[n - 1 - n / 200];
  const float extent = top - bottom;
  if (!(extent >= 1.0f)) return head;  // not a standing person (or not in metres)
  // The head slab: the top 13% of the extent. Its points projected off the up axis.
  const float slab = top - 0.13f * extent;
  std::vector<float> across[3];
  for (size_t i = 0; i < n; ++i) {
    if (h[i] < slab || h[i] > top) continue;
    for (int k = 0; k < 3; ++k) across[k].push_back(subject.positions[i * 3 + k] - h[i] * up[k]);
  }
  if (across[0].size() < 20) return head;
  // Per axis the median across the slab, at 8.5% of the extent below the top (below the
  // slab's middle: hair raises the top).
  const float level = top - 0.085f * extent;
  for (int k = 0; k < 3; ++k) {
    std::vector<float>& a = across[k];
    std::nth_element(a.begin(), a.begin() + a.size() / 2, a.end());
    head.center[k] = a[a.size() / 2] + level * up[k];
  }
  head.radius = 0.1f * extent;
  head.subject_height = extent;
  head.found = true;
  return head;
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

namespace {

std::string join(const std::string& dir, const std::string& file) {
  if (file.empty() || file[0] == '/') return file;
  return dir.empty() || dir.back() == '/' ? dir + file : dir + "/" + file;
}

uint64_t cell_key(int64_t x, int64_t y, int64_t z) {
  return (uint64_t(x) & 0x1fffffull) | (uint64_t(y) & 0x1fffffull) << 21 | (uint64_t(z) & 0x1fffffull) << 42;
}

// 10 bits of v spread to every third bit (Morton order).
uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

}  // namespace

Dataset load_dataset(const std::string& directory, uint32_t target_width) {
  const std::vector<uint8_t> text = read_file(join(directory, "transforms.json"));
  const detail::Json root = detail::parse_json(std::string(text.begin(), text.end()));
  const detail::Json* frames = root.find("frames");
  if (frames == nullptr || frames->type != detail::Json::Type::Array || frames->array.empty())
    throw std::runtime_error("transforms.json has no frames");
  const double src_w = root.number_or("w", 0), src_h = root.number_or("h", 0);
  const double fl_x = root.number_or("fl_x", 0), fl_y = root.number_or("fl_y", fl_x);
  if (src_w <= 0 || src_h <= 0 || fl_x <= 0) throw std::runtime_error("transforms.json has no w/h/fl_x");
  Dataset ds;
  if (const detail::Json* lab = root.find("gsplat_lab")) {
    const detail::Json* up = lab->find("world_up");
    if (up != nullptr && up->array.size() == 3) {
      double len = 0.0;
      for (const detail::Json& v : up->array) len += v.number * v.number;
      len = std::sqrt(len);
      if (len > 0.0)
        for (int k = 0; k < 3; ++k) ds.world_up[k] = float(up->array[size_t(k)].number / len);
    }
  }
  std::string trimmed = directory;
  while (trimmed.size() > 1 && trimmed.back() == '/') trimmed.pop_back();
  const size_t slash = trimmed.find_last_of('/');
  ds.name = slash == std::string::npos ? trimmed : trimmed.substr(slash + 1);
  // The short side becomes target_width (never enlarged).
  const double s = std::min(1.0, double(target_width) / std::min(src_w, src_h));
  ds.width = uint32_t(std::lround(src_w * s));
  ds.height = uint32_t(std::lround(src_h * s));
  ds.fx = float(fl_x * s);
  ds.fy = float(fl_y * s);
  ds.cx = float(root.number_or("cx", src_w / 2) * s);
  ds.cy = float(root.number_or("cy", src_h / 2) * s);
  const size_t n = frames->array.size();
  std::vector<DatasetFrame> all(n);
  std::vector<std::string> images(n), masks(n);
  for (size_t i = 0; i < n; ++i) {
    const detail::Json& f = frames->array[i];
    images[i] = f.string_or("file_path", "");
    if (images[i].empty()) throw std::runtime_error("a frame has no file_path");
    all[i].name = images[i];
    const detail::Json* m = f.find("transform_matrix");
    if (m == nullptr || m->array.size() != 4) throw std::runtime_error("a frame has no 4x4 transform_matrix");
    for (int r = 0; r < 4; ++r) {
      if (m->array[size_t(r)].array.size() != 4) throw std::runtime_error("transform_matrix is not 4x4");
      for (int col = 0; col < 4; ++col) all[i].c2w[r * 4 + col] = float(m->array[size_t(r)].array[size_t(col)].number);
    }
    masks[i] = f.string_or("mask_path", "");
    all[i].holdout = i % 8 == 0;
  }
  ds.has_masks = std::all_of(masks.begin(), masks.end(), [](const std::string& p) { return !p.empty(); });
  for (size_t i = 0; i < n; ++i) {
    DatasetFrame& frame = all[i];
    try {
      const detail::Image img = detail::decode_image(read_file(join(directory, images[i])), 4);
      if (img.width != uint32_t(src_w) || img.height != uint32_t(src_h))
        throw std::runtime_error("size differs from transforms.json");
      frame.rgba = detail::resize_area(img.data.data(), img.width, img.height, 4, ds.width, ds.height);
      if (ds.has_masks) {
        const detail::Image mask = detail::decode_image(read_file(join(directory, masks[i])), 1);
        const std::vector<uint8_t> m = detail::resize_area(mask.data.data(), mask.width, mask.height, 1, ds.width, ds.height);
        for (size_t p = 0; p < m.size(); ++p) frame.rgba[p * 4 + 3] = m[p];
      } else {
        for (size_t p = 0; p < size_t(ds.width) * ds.height; ++p) frame.rgba[p * 4 + 3] = 255;
      }
      ds.frames.push_back(std::move(frame));
    } catch (const std::exception& e) {
      ds.skipped.push_back(images[i] + ": " + e.what());
    }
  }
  if (ds.frames.size() < 2 || ds.frames.size() * 2 < n)
    throw std::runtime_error("too few readable frames (" + std::to_string(ds.frames.size()) + "/" + std::to_string(n) +
                             ")" + (ds.skipped.empty() ? std::string() : ": " + ds.skipped.front()));
  const std::string ply = root.string_or("ply_file_path", "");
  if (!ply.empty()) {
    const std::vector<uint8_t> bytes = read_file(join(directory, ply));
    const PlyVertices v(bytes.data(), bytes.size());
    const int x = v.find("x"), y = v.find("y"), z = v.find("z"), r = v.find("red"), g = v.find("green"),
              b = v.find("blue");
    if (x < 0 || y < 0 || z < 0) throw std::runtime_error("point cloud PLY has no x/y/z");
    ds.points.resize(size_t(v.count()) * 3);
    ds.point_colors.assign(size_t(v.count()) * 3, 128);
    for (uint64_t i = 0; i < v.count(); ++i) {
      ds.points[size_t(i) * 3 + 0] = v.value(i, x);
      ds.points[size_t(i) * 3 + 1] = v.value(i, y);
      ds.points[size_t(i) * 3 + 2] = v.value(i, z);
      if (r >= 0 && g >= 0 && b >= 0) {
        ds.point_colors[size_t(i) * 3 + 0] = uint8_t(v.value(i, r));
        ds.point_colors[size_t(i) * 3 + 1] = uint8_t(v.value(i, g));
        ds.point_colors[size_t(i) * 3 + 2] = uint8_t(v.value(i, b));
      }
    }
  }
  compute_camera_bounds(ds);
  return ds;
}

SplatScene initialize_gaussians(const Dataset& ds, const InitOptions& o, InitStats* stats) {
  std::vector<float> pts, cols;  // colours in [0, 1]
  std::string source = "points";
  if (!ds.points.empty()) {
    pts = ds.points;
    for (uint8_t c : ds.point_colors) cols.push_back(float(c) / 255.0f);
  } else {
    source = "random";  // uniform in a ball of half the camera extent around the cameras' centre
    std::mt19937 rng(o.seed);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f);
    const float radius = 0.5f * ds.camera_extent;
    for (uint32_t i = 0; i < o.max_gaussians; ++i) {
      float p[3];
      do
        for (float& v : p) v = u(rng);
      while (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > 1.0f);
      for (int k = 0; k < 3; ++k) {
        pts.push_back(ds.camera_center[k] + radius * p[k]);
        cols.push_back(0.5f);
      }
    }
  }
  const size_t raw = pts.size() / 3;
  if (raw == 0) throw std::runtime_error("initialize_gaussians: no points");
  float lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = INFINITY;
    hi[k] = -INFINITY;
  }
  for (size_t i = 0; i < raw; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pts[i * 3 + k]);
      hi[k] = std::max(hi[k], pts[i * 3 + k]);
    }
  // The span without strays: the diagonal of the 0.5%..99.5% box.
  float extent = 1e-6f;
  {
    std::vector<float> axis(raw);
    double e2 = 0.0;
    for (int k = 0; k < 3; ++k) {
      for (size_t i = 0; i < raw; ++i) axis[i] = pts[i * 3 + k];
      const size_t a = raw / 200, b = raw - 1 - raw / 200;
      std::nth_element(axis.begin(), axis.begin() + long(a), axis.end());
      const float low = axis[a];
      std::nth_element(axis.begin(), axis.begin() + long(b), axis.end());
      e2 += double(axis[b] - low) * double(axis[b] - low);
    }
    extent += float(std::sqrt(e2));
  }
  auto cell_of = [&](const float* p, float cell, int64_t c[3]) {
    for (int k = 0; k < 3; ++k) c[k] = int64_t(std::floor((p[k] - lo[k]) / cell));
  };
  auto occupied = [&](const std::vector<float>& p, float cell) {
    std::vector<uint64_t> keys(p.size() / 3);
    for (size_t i = 0; i < keys.size(); ++i) {
      int64_t c[3];
      cell_of(&p[i * 3], cell, c);
      keys[i] = cell_key(c[0], c[1], c[2]);
    }
    std::sort(keys.begin(), keys.end());
    return size_t(std::unique(keys.begin(), keys.end()) - keys.begin());
  };
  // The cell size whose occupied-cell count lands just under `target` (log-space bisection;
  // the large end is doubled first until it is under, so the budget always holds).
  auto cell_for = [&](const std::vector<float>& p, size_t target) {
    float small = extent * 1e-4f, large = extent * 0.1f;
    for (int it = 0; it < 40 && occupied(p, large) > target; ++it) large *= 2.0f;
    for (int it = 0; it < 12; ++it) {
      const float mid = std::sqrt(small * large);
      (occupied(p, mid) > target ? small : large) = mid;
    }
    return large;
  };
  float voxel = 0.0f;
  if (raw > o.max_gaussians) {
    voxel = cell_for(pts, o.max_gaussians);
    struct Acc {
      double p[3] = {0, 0, 0}, c[3] = {0, 0, 0};
      uint32_t n = 0;
    };
    std::unordered_map<uint64_t, Acc> cells;
    for (size_t i = 0; i < raw; ++i) {
      int64_t c[3];
      cell_of(&pts[i * 3], voxel, c);
      Acc& a = cells[cell_key(c[0], c[1], c[2])];
      for (int k = 0; k < 3; ++k) {
        a.p[k] += pts[i * 3 + k];
        a.c[k] += cols[i * 3 + k];
      }
      ++a.n;
    }
    std::vector<float> mp, mc;
    for (const auto& kv : cells)
      for (int k = 0; k < 3; ++k) {
        mp.push_back(float(kv.second.p[k] / kv.second.n));
        mc.push_back(float(kv.second.c[k] / kv.second.n));
      }
    pts.swap(mp);
    cols.swap(mc);
  }
  const size_t n = pts.size() / 3;
  // Morton order: neighbours in space are neighbours in memory.
  {
    std::vector<std::pair<uint32_t, uint32_t>> order(n);
    for (size_t i = 0; i < n; ++i) {
      uint32_t code = 0;
      for (int k = 0; k < 3; ++k) {
        const float span = std::max(hi[k] - lo[k], 1e-6f);
        code |= spread3(uint32_t(std::min(std::max((pts[i * 3 + k] - lo[k]) / span, 0.0f), 1.0f) * 1023.0f)) << k;
      }
      order[i] = {code, uint32_t(i)};
    }
    std::sort(order.begin(), order.end());
    std::vector<float> p2(pts.size()), c2(cols.size());
    for (size_t j = 0; j < n; ++j)
      for (int k = 0; k < 3; ++k) {
        p2[j * 3 + k] = pts[size_t(order[j].second) * 3 + k];
        c2[j * 3 + k] = cols[size_t(order[j].second) * 3 + k];
      }
    pts.swap(p2);
    cols.swap(c2);
  }
  // Scales: mean distance to the 3 nearest neighbours, found in a grid of about two
  // points' spacing.
  const float cell = 2.0f * (voxel > 0.0f ? voxel : cell_for(pts, std::max<size_t>(n / 2, 1)));
  std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
  for (uint32_t i = 0; i < n; ++i) {
    int64_t c[3];
    cell_of(&pts[size_t(i) * 3], cell, c);
    grid[cell_key(c[0], c[1], c[2])].push_back(i);
  }
  SplatScene scene;
  scene.convention = AxisConvention::RUB;
  scene.resize(uint32_t(n), 0);
  const float logit = std::log(o.initial_opacity / (1.0f - o.initial_opacity));
  constexpr float kC0 = 0.28209479177387814f;  // SH DC basis value
  for (uint32_t i = 0; i < n; ++i) {
    const float* p = &pts[size_t(i) * 3];
    int64_t c[3];
    cell_of(p, cell, c);
    float best[3] = {INFINITY, INFINITY, INFINITY};
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const auto it = grid.find(cell_key(c[0] + dx, c[1] + dy, c[2] + dz));
          if (it == grid.end()) continue;
          for (uint32_t j : it->second) {
            if (j == i) continue;
            const float* q = &pts[size_t(j) * 3];
            const float d2 = (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]);
            if (d2 < best[2]) {
              best[2] = d2;
              std::sort(best, best + 3);
            }
          }
        }
    float mean = 0.0f;
    int found = 0;
    for (float d2 : best)
      if (std::isfinite(d2)) {
        mean += std::sqrt(d2);
        ++found;
      }
    const float scale = std::min(std::max(found > 0 ? mean / float(found) : cell, 1e-4f * extent), 0.02f * extent);
    for (int k = 0; k < 3; ++k) {
      scene.positions[size_t(i) * 3 + k] = p[k];
      scene.log_scales[size_t(i) * 3 + k] = std::log(scale);
      scene.sh_dc[size_t(i) * 3 + k] = (cols[size_t(i) * 3 + k] - 0.5f) / kC0;
    }
    scene.rotations[size_t(i) * 4] = 1.0f;
    scene.opacity_logits[i] = logit;
  }
  if (stats != nullptr) {
    stats->source = source;
    stats->raw_points = raw;
    stats->voxel_size = voxel;
  }
  return scene;
}

}  // namespace gs
