// Datasets: camera bounds and cameras (engine/src/dataset.cpp:60-83, 226-250) and
// synthetic orbit captures rendered through libgs_cuda.
#include "gs/dataset.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <array>
#include <random>
#include <stdexcept>

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
  const double depth_unit = root.number_or("depth_unit_scale_factor", 0.001);  // metres per depth sample
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
  std::vector<std::string> images(n), masks(n), depths(n), confidences(n);
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
    depths[i] = f.string_or("depth_file_path", "");
    confidences[i] = f.string_or("depth_confidence_path", "");
    all[i].holdout = i % 8 == 0;
  }
  ds.has_masks = std::all_of(masks.begin(), masks.end(), [](const std::string& p) { return !p.empty(); });
  ds.has_depth = std::any_of(depths.begin(), depths.end(), [](const std::string& p) { return !p.empty(); });
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
    } catch (const std::exception& e) {
      ds.skipped.push_back(images[i] + ": " + e.what());
      continue;
    }
    // Depth is optional per frame: one that cannot be read just adds no points.
    if (!depths[i].empty()) {
      try {
        const detail::Depth16 d = detail::decode_depth16(read_file(join(directory, depths[i])));
        frame.depth.resize(d.data.size());
        for (size_t p = 0; p < d.data.size(); ++p) frame.depth[p] = float(double(d.data[p]) * depth_unit);
        frame.depth_width = d.width;
        frame.depth_height = d.height;
        if (!confidences[i].empty()) {
          detail::Image c = detail::decode_image(read_file(join(directory, confidences[i])), 1);
          if (c.width == d.width && c.height == d.height) frame.depth_confidence = std::move(c.data);
        }
      } catch (const std::exception&) {
        frame.depth.clear();
        frame.depth_confidence.clear();
        frame.depth_width = frame.depth_height = 0;
      }
    }
    ds.frames.push_back(std::move(frame));
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

namespace {

// A coloured point set: xyz and rgb (0..1), three floats each per point.
struct Cloud {
  std::vector<float> xyz, rgb;
  size_t size() const { return xyz.size() / 3; }
};

// The training frames' depth samples as world points, coloured by the frame's pixel there.
Cloud depth_cloud(const Dataset& ds, const InitOptions& o) {
  Cloud c;
  const float floor_conf = std::clamp(o.min_confidence, 0.0f, 1.0f) * 255.0f;
  const bool subject = o.subject_only && ds.has_masks;
  for (const DatasetFrame& f : ds.frames) {
    if (f.holdout || f.depth.empty()) continue;
    const Camera cam = dataset_camera(ds, f);
    for (uint32_t v = 0; v < f.depth_height; ++v)
      for (uint32_t u = 0; u < f.depth_width; ++u) {
        const size_t at = size_t(v) * f.depth_width + u;
        const double z = f.depth[at];
        if (!(z > 0.0)) continue;
        if (!f.depth_confidence.empty() && float(f.depth_confidence[at]) < floor_conf) continue;
        // The sample's centre in training pixels, and the pixel it lands in.
        const double px = (u + 0.5) * cam.width / f.depth_width, py = (v + 0.5) * cam.height / f.depth_height;
        const uint32_t ix = std::min(cam.width - 1, uint32_t(px)), iy = std::min(cam.height - 1, uint32_t(py));
        const uint8_t* rgba = &f.rgba[(size_t(iy) * cam.width + ix) * 4];
        if (subject && rgba[3] < 128) continue;
        // OpenCV camera coordinates; the OpenGL camera-to-world takes (x, -y, -z).
        const double x = (px - cam.cx) / cam.fx * z, y = (py - cam.cy) / cam.fy * z;
        for (int r = 0; r < 3; ++r)
          c.xyz.push_back(float(f.c2w[r * 4] * x - f.c2w[r * 4 + 1] * y - f.c2w[r * 4 + 2] * z + f.c2w[r * 4 + 3]));
        for (int k = 0; k < 3; ++k) c.rgb.push_back(float(rgba[k]) / 255.0f);
      }
  }
  return c;
}

Cloud random_cloud(const Dataset& ds, uint32_t count, uint32_t seed) {
  Cloud c;
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> u(-1.0f, 1.0f);
  const float radius = 0.5f * ds.camera_extent;
  while (c.size() < count) {
    const float p[3] = {u(rng), u(rng), u(rng)};
    if (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > 1.0f) continue;  // inside the unit ball
    for (int k = 0; k < 3; ++k) {
      c.xyz.push_back(ds.camera_center[k] + radius * p[k]);
      c.rgb.push_back(0.5f);
    }
  }
  return c;
}

// The diagonal of the box between each axis's 0.5% and 99.5% order statistics: the span
// of the points without strays (depth smeared off an edge, flyers).
float robust_extent(const std::vector<float>& xyz) {
  const size_t n = xyz.size() / 3;
  std::vector<float> axis(n);
  double d2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    for (size_t i = 0; i < n; ++i) axis[i] = xyz[i * 3 + k];
    const size_t lo = n / 200, hi = n - 1 - n / 200;
    std::nth_element(axis.begin(), axis.begin() + long(lo), axis.end());
    const float a = axis[lo];
    std::nth_element(axis.begin(), axis.begin() + long(hi), axis.end());
    d2 += double(axis[hi] - a) * double(axis[hi] - a);
  }
  return float(std::sqrt(d2)) + 1e-6f;
}

// Grid cells of size `cell` from `origin`, 21 bits per axis in one 63-bit key.
struct Grid {
  float origin[3];
  float cell;
  uint64_t key(const float* p) const {
    uint64_t out = 0;
    for (int k = 0; k < 3; ++k) {
      const double c = std::floor((double(p[k]) - origin[k]) / cell);
      out |= (uint64_t(int64_t(std::clamp(c, 0.0, double((1 << 21) - 1)))) & 0x1fffffu) << (21 * k);
    }
    return out;
  }
};

// (cell key, point) of every point, sorted by key: a cell's points are one run.
std::vector<std::pair<uint64_t, uint32_t>> by_cell(const std::vector<float>& xyz, const Grid& g) {
  std::vector<std::pair<uint64_t, uint32_t>> keyed(xyz.size() / 3);
  for (size_t i = 0; i < keyed.size(); ++i) keyed[i] = {g.key(&xyz[i * 3]), uint32_t(i)};
  std::sort(keyed.begin(), keyed.end());
  return keyed;
}

size_t occupied(const std::vector<float>& xyz, const Grid& g) {
  std::vector<uint64_t> keys(xyz.size() / 3);
  for (size_t i = 0; i < keys.size(); ++i) keys[i] = g.key(&xyz[i * 3]);
  std::sort(keys.begin(), keys.end());
  return size_t(std::unique(keys.begin(), keys.end()) - keys.begin());
}

// A cell size whose occupied-cell count is at most `budget` and close under it. The count
// falls with the cell size roughly as a power law (size^-D, D the points' dimension), so
// the size is found by false position on log(count) against log(size), kept inside a
// bracket [small: count over budget, large: count within it] that every probe narrows.
float fit_cell(const std::vector<float>& xyz, Grid g, float extent, size_t budget) {
  auto count_at = [&](double cell) {
    g.cell = float(cell);
    return double(std::max<size_t>(occupied(xyz, g), 1));
  };
  double small = extent * 1e-4, large = extent;
  double n_small = count_at(small), n_large = count_at(large);
  if (n_small <= double(budget)) return float(small);
  for (int i = 0; i < 60 && n_large > double(budget); ++i) n_large = count_at(large *= 2.0);
  const double target = std::log(0.97 * double(budget));
  for (int round = 0; round < 24; ++round) {
    if (n_large >= 0.9 * double(budget) || large / small < 1.01) break;
    // Where the line through the bracket's ends in log-log space meets the target, kept
    // away from the ends (else the geometric middle).
    const double ls = std::log(small), ll = std::log(large);
    const double ys = std::log(n_small), yl = std::log(n_large);
    double x = ys > yl ? ls + (ys - target) * (ll - ls) / (ys - yl) : 0.5 * (ls + ll);
    const double margin = 0.05 * (ll - ls);
    if (!(x > ls + margin && x < ll - margin)) x = 0.5 * (ls + ll);
    const double cell = std::exp(x), n = count_at(cell);
    if (n > double(budget)) {
      small = cell;
      n_small = n;
    } else {
      large = cell;
      n_large = n;
    }
  }
  return float(large);
}

// The points of each occupied cell replaced by their mean (position and colour).
Cloud merge_cells(const Cloud& in, const Grid& g) {
  const auto keyed = by_cell(in.xyz, g);
  Cloud out;
  for (size_t a = 0; a < keyed.size();) {
    size_t b = a;
    double sum[6] = {0, 0, 0, 0, 0, 0};
    for (; b < keyed.size() && keyed[b].first == keyed[a].first; ++b)
      for (int k = 0; k < 3; ++k) {
        sum[k] += in.xyz[size_t(keyed[b].second) * 3 + k];
        sum[3 + k] += in.rgb[size_t(keyed[b].second) * 3 + k];
      }
    const double n = double(b - a);
    for (int k = 0; k < 3; ++k) {
      out.xyz.push_back(float(sum[k] / n));
      out.rgb.push_back(float(sum[3 + k] / n));
    }
    a = b;
  }
  return out;
}

// The points reordered along a Z-order (Morton) curve over their bounding box, 10 bits per
// axis: points near in space are near in memory.
Cloud morton_sorted(const Cloud& in) {
  const size_t n = in.size();
  float lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = INFINITY;
    hi[k] = -INFINITY;
  }
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], in.xyz[i * 3 + k]);
      hi[k] = std::max(hi[k], in.xyz[i * 3 + k]);
    }
  std::vector<std::pair<uint32_t, uint32_t>> code(n);
  for (size_t i = 0; i < n; ++i) {
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      const float t = (in.xyz[i * 3 + k] - lo[k]) / std::max(hi[k] - lo[k], 1e-6f);
      q[k] = uint32_t(std::clamp(t, 0.0f, 1.0f) * 1023.0f);
    }
    uint32_t z = 0;
    for (int bit = 9; bit >= 0; --bit)
      for (int k = 2; k >= 0; --k) z = z << 1 | ((q[k] >> bit) & 1u);
    code[i] = {z, uint32_t(i)};
  }
  std::sort(code.begin(), code.end());
  Cloud out;
  out.xyz.reserve(in.xyz.size());
  out.rgb.reserve(in.rgb.size());
  for (const auto& c : code)
    for (int k = 0; k < 3; ++k) {
      out.xyz.push_back(in.xyz[size_t(c.second) * 3 + k]);
      out.rgb.push_back(in.rgb[size_t(c.second) * 3 + k]);
    }
  return out;
}

// A k-d tree over points (median splits on the widest axis) answering "the k nearest
// other points" by branch-and-bound.
class KdTree {
 public:
  explicit KdTree(const std::vector<float>& xyz) : xyz_(xyz), index_(xyz.size() / 3) {
    for (size_t i = 0; i < index_.size(); ++i) index_[i] = uint32_t(i);
    build(0, 0, index_.size());
  }
  // Squared distances to the (up to) 3 nearest points other than point `self`, ascending.
  std::array<float, 3> nearest3(uint32_t self) const {
    std::array<float, 3> best{INFINITY, INFINITY, INFINITY};
    search(0, 0, index_.size(), &xyz_[size_t(self) * 3], self, best);
    return best;
  }

 private:
  struct Split {
    int axis;
    float value;
  };
  // Node `node` holds points [a, b) of index_; its children are 2 node + 1 and 2 node + 2.
  void build(size_t node, size_t a, size_t b) {
    if (b - a <= kLeaf) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = a; i < b; ++i)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], xyz_[size_t(index_[i]) * 3 + k]);
        hi[k] = std::max(hi[k], xyz_[size_t(index_[i]) * 3 + k]);
      }
    int axis = 0;
    for (int k = 1; k < 3; ++k)
      if (hi[k] - lo[k] > hi[axis] - lo[axis]) axis = k;
    const size_t mid = (a + b) / 2;
    std::nth_element(index_.begin() + long(a), index_.begin() + long(mid), index_.begin() + long(b),
                     [&](uint32_t i, uint32_t j) { return xyz_[size_t(i) * 3 + axis] < xyz_[size_t(j) * 3 + axis]; });
    if (splits_.size() <= node) splits_.resize(2 * node + 1);
    splits_[node] = {axis, xyz_[size_t(index_[mid]) * 3 + axis]};
    build(2 * node + 1, a, mid);
    build(2 * node + 2, mid, b);
  }
  void search(size_t node, size_t a, size_t b, const float* q, uint32_t self, std::array<float, 3>& best) const {
    if (b - a <= kLeaf) {
      for (size_t i = a; i < b; ++i) {
        if (index_[i] == self) continue;
        const float* p = &xyz_[size_t(index_[i]) * 3];
        const float d2 = (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]);
        if (d2 < best[2]) {
          best[2] = d2;
          std::sort(best.begin(), best.end());
        }
      }
      return;
    }
    const Split s = splits_[node];
    const size_t mid = (a + b) / 2;
    const float gap = q[s.axis] - s.value;
    const bool left_first = gap < 0.0f;
    const size_t near = left_first ? 2 * node + 1 : 2 * node + 2, far = left_first ? 2 * node + 2 : 2 * node + 1;
    search(near, left_first ? a : mid, left_first ? mid : b, q, self, best);
    if (gap * gap < best[2]) search(far, left_first ? mid : a, left_first ? b : mid, q, self, best);
  }
  static constexpr size_t kLeaf = 16;
  const std::vector<float>& xyz_;
  std::vector<uint32_t> index_;
  std::vector<Split> splits_;
};

}  // namespace

SplatScene initialize_gaussians(const Dataset& ds, const InitOptions& o, InitStats* stats) {
  Cloud cloud;
  std::string source;
  if (ds.has_depth) {
    cloud = depth_cloud(ds, o);
    source = "depth";
  }
  if (cloud.size() == 0 && !ds.points.empty()) {
    cloud.xyz = ds.points;
    for (uint8_t c : ds.point_colors) cloud.rgb.push_back(float(c) / 255.0f);
    source = "points";
  }
  if (cloud.size() == 0) {
    cloud = random_cloud(ds, o.max_gaussians, o.seed);
    source = "random";
  }
  const size_t raw = cloud.size();
  if (raw == 0) throw std::runtime_error("initialize_gaussians: no points");
  const float extent = robust_extent(cloud.xyz);
  float voxel = 0.0f;
  if (raw > o.max_gaussians) {
    Grid g{{INFINITY, INFINITY, INFINITY}, 0.0f};
    for (size_t i = 0; i < raw; ++i)
      for (int k = 0; k < 3; ++k) g.origin[k] = std::min(g.origin[k], cloud.xyz[i * 3 + k]);
    voxel = fit_cell(cloud.xyz, g, extent, std::max<size_t>(o.max_gaussians, 1));
    g.cell = voxel;
    cloud = merge_cells(cloud, g);
  }
  cloud = morton_sorted(cloud);
  const size_t n = cloud.size();
  const KdTree tree(cloud.xyz);
  SplatScene scene;
  scene.convention = AxisConvention::RUB;
  scene.resize(uint32_t(n), 0);
  const float logit = std::log(o.initial_opacity / (1.0f - o.initial_opacity));
  constexpr float kC0 = 0.28209479177387814f;  // the SH DC basis value
  for (size_t i = 0; i < n; ++i) {
    const std::array<float, 3> d2 = tree.nearest3(uint32_t(i));
    double sum = 0.0;
    int found = 0;
    for (float v : d2)
      if (std::isfinite(v)) {
        sum += std::sqrt(double(v));
        ++found;
      }
    const float mean = found > 0 ? float(sum / found) : 0.01f * extent;
    const float scale = std::clamp(mean, 1e-4f * extent, 0.02f * extent);
    for (int k = 0; k < 3; ++k) {
      scene.positions[i * 3 + k] = cloud.xyz[i * 3 + k];
      scene.log_scales[i * 3 + k] = std::log(scale);
      scene.sh_dc[i * 3 + k] = (cloud.rgb[i * 3 + k] - 0.5f) / kC0;
    }
    scene.rotations[i * 4] = 1.0f;
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
