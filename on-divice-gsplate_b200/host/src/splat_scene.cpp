// Host scenes: PLY reading and writing, axis conversion, random scenes.
// Interface of engine/include/gs/splat_scene.h; formats of engine/src/splat_scene.cpp:264-365
// (the standard 3DGS PLY: x y z nx ny nz f_dc_0..2 f_rest_* opacity scale_0..2 rot_0..3,
// f_rest channel-major).
#include "gs/splat_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iterator>
#include <random>
#include <sstream>
#include <stdexcept>

namespace gs {

namespace {

struct ScalarType {
  const char* names[2];
  size_t bytes;
};
// PLY scalar types (both the short and the sized names).
constexpr ScalarType kTypes[] = {
    {{"char", "int8"}, 1},   {{"uchar", "uint8"}, 1},   {{"short", "int16"}, 2},  {{"ushort", "uint16"}, 2},
    {{"int", "int32"}, 4},   {{"uint", "uint32"}, 4},   {{"float", "float32"}, 4}, {{"double", "float64"}, 8},
};

int type_index(const std::string& name) {
  for (int t = 0; t < int(std::size(kTypes)); ++t)
    if (name == kTypes[t].names[0] || name == kTypes[t].names[1]) return t;
  return -1;
}

template <typename T>
T load_le(const uint8_t* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}

int degree_for_rest(int coeffs) {
  for (int d = 0; d <= 3; ++d)
    if (sh_rest_coeffs(d) == coeffs) return d;
  return -1;
}

}  // namespace

int sh_rest_coeffs(int degree) { return degree <= 0 ? 0 : (degree + 1) * (degree + 1) - 1; }

void SplatScene::resize(uint32_t n, int degree) {
  count = n;
  sh_degree = degree;
  positions.assign(size_t(n) * 3, 0.0f);
  log_scales.assign(size_t(n) * 3, 0.0f);
  rotations.assign(size_t(n) * 4, 0.0f);
  opacity_logits.assign(n, 0.0f);
  sh_dc.assign(size_t(n) * 3, 0.0f);
  sh_rest.assign(size_t(n) * sh_rest_coeffs(degree) * 3, 0.0f);
}

SceneBounds compute_bounds(const SplatScene& scene) {
  SceneBounds b{{0.0f, 0.0f, 0.0f}, 1.0f};
  if (scene.count == 0) return b;
  std::vector<float> axis(scene.count);
  for (int k = 0; k < 3; ++k) {
    for (uint32_t i = 0; i < scene.count; ++i) axis[i] = scene.positions[size_t(i) * 3 + k];
    std::nth_element(axis.begin(), axis.begin() + axis.size() / 2, axis.end());
    b.center[k] = axis[axis.size() / 2];
  }
  for (uint32_t i = 0; i < scene.count; ++i) {
    float d2 = 0.0f;
    for (int k = 0; k < 3; ++k) {
      const float d = scene.positions[size_t(i) * 3 + k] - b.center[k];
      d2 += d * d;
    }
    axis[i] = std::sqrt(d2);
  }
  const size_t q = std::min(axis.size() - 1, size_t(0.9 * double(axis.size())));
  std::nth_element(axis.begin(), axis.begin() + q, axis.end());
  b.radius = std::max(axis[q], 1e-3f);
  return b;
}

PlyVertices::PlyVertices(const uint8_t* data, size_t size) {
  const char kEnd[] = "end_header\n";
  const uint8_t* end = std::search(data, data + size, kEnd, kEnd + sizeof(kEnd) - 1);
  if (size < 4 || std::memcmp(data, "ply", 3) != 0 || end == data + size)
    throw std::runtime_error("not a PLY file (no ply magic or end_header)");
  std::istringstream header(std::string(reinterpret_cast<const char*>(data), size_t(end - data)));
  std::string line;
  bool in_vertex = false, seen_vertex = false;
  size_t skip_before = 0;  // bytes of elements before the vertex element (fixed-size ones only)
  uint64_t pending_count = 0;
  size_t pending_stride = 0;
  bool pending_list = false;
  auto close_element = [&]() {
    if (!in_vertex && !seen_vertex && pending_count > 0) {
      if (pending_list) throw std::runtime_error("PLY: list elements before the vertex element are not supported");
      skip_before += size_t(pending_count) * pending_stride;
    }
  };
  while (std::getline(header, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream words(line);
    std::string word;
    words >> word;
    if (word == "format") {
      std::string fmt;
      words >> fmt;
      if (fmt != "binary_little_endian") throw std::runtime_error("PLY: only binary_little_endian is supported");
    } else if (word == "element") {
      close_element();
      std::string name;
      uint64_t n = 0;
      words >> name >> n;
      in_vertex = name == "vertex";
      if (in_vertex) {
        seen_vertex = true;
        count_ = n;
      }
      pending_count = in_vertex ? 0 : n;
      pending_stride = 0;
      pending_list = false;
    } else if (word == "property") {
      std::string type, name;
      words >> type;
      if (type == "list") {
        if (in_vertex) throw std::runtime_error("PLY: list properties on vertices are not supported");
        pending_list = true;
        continue;
      }
      words >> name;
      const int t = type_index(type);
      if (t < 0) throw std::runtime_error("PLY: unknown property type " + type);
      if (in_vertex) {
        properties_.push_back({name, t, stride_});
        stride_ += kTypes[t].bytes;
      } else {
        pending_stride += kTypes[t].bytes;
      }
    }
  }
  if (!seen_vertex) throw std::runtime_error("PLY: no vertex element");
  base_ = end + (sizeof(kEnd) - 1) + skip_before;
  const size_t available = size_t((data + size) - base_);
  if (stride_ == 0 || count_ > available / stride_) throw std::runtime_error("PLY: vertex data is truncated");
}

int PlyVertices::find(const std::string& name) const {
  for (size_t i = 0; i < properties_.size(); ++i)
    if (properties_[i].name == name) return int(i);
  return -1;
}

float PlyVertices::value(uint64_t vertex, int property) const {
  const Property& p = properties_.at(size_t(property));
  const uint8_t* at = base_ + size_t(vertex) * stride_ + p.offset;
  switch (p.type) {
    case 0: return float(load_le<int8_t>(at));
    case 1: return float(load_le<uint8_t>(at));
    case 2: return float(load_le<int16_t>(at));
    case 3: return float(load_le<uint16_t>(at));
    case 4: return float(load_le<int32_t>(at));
    case 5: return float(load_le<uint32_t>(at));
    case 6: return load_le<float>(at);
    default: return float(load_le<double>(at));
  }
}

SplatScene load_ply(const uint8_t* data, size_t size) {
  const PlyVertices ply(data, size);
  auto require = [&](const std::string& name) {
    const int index = ply.find(name);
    if (index < 0) throw std::runtime_error("not a gaussian splat PLY (no " + name + " property)");
    return index;
  };
  int rest_count = 0;
  while (ply.find("f_rest_" + std::to_string(rest_count)) >= 0) ++rest_count;
  const int file_coeffs = rest_count / 3;
  const int file_degree = rest_count % 3 == 0 ? degree_for_rest(file_coeffs) : -1;
  if (file_degree < 0) throw std::runtime_error("PLY: the f_rest count fits no SH degree up to 3");
  const int xyz[3] = {require("x"), require("y"), require("z")};
  const int dc[3] = {require("f_dc_0"), require("f_dc_1"), require("f_dc_2")};
  const int opacity = require("opacity");
  const int scale[3] = {require("scale_0"), require("scale_1"), require("scale_2")};
  const int rot[4] = {require("rot_0"), require("rot_1"), require("rot_2"), require("rot_3")};
  std::vector<int> rest(static_cast<size_t>(rest_count));
  for (int i = 0; i < rest_count; ++i) rest[size_t(i)] = ply.find("f_rest_" + std::to_string(i));
  if (ply.count() > 0xffffffffull) throw std::runtime_error("PLY: too many vertices");
  SplatScene scene;
  scene.convention = AxisConvention::RDF;
  scene.resize(uint32_t(ply.count()), file_degree);
  for (uint32_t i = 0; i < scene.count; ++i) {
    for (int k = 0; k < 3; ++k) {
      scene.positions[size_t(i) * 3 + k] = ply.value(i, xyz[k]);
      scene.sh_dc[size_t(i) * 3 + k] = ply.value(i, dc[k]);
      scene.log_scales[size_t(i) * 3 + k] = ply.value(i, scale[k]);
    }
    for (int k = 0; k < 4; ++k) scene.rotations[size_t(i) * 4 + k] = ply.value(i, rot[k]);
    scene.opacity_logits[i] = ply.value(i, opacity);
    for (int j = 0; j < file_coeffs; ++j)
      for (int c = 0; c < 3; ++c)
        scene.sh_rest[(size_t(i) * file_coeffs + j) * 3 + c] = ply.value(i, rest[size_t(c * file_coeffs + j)]);
  }
  return scene;
}

SplatScene load_splat_file(const uint8_t* data, size_t size) {
  if (size >= 3 && std::memcmp(data, "ply", 3) == 0) return load_ply(data, size);
  throw std::runtime_error("not a PLY splat file");
}

std::vector<uint8_t> save_ply(const SplatScene& scene) {
  const int coeffs = sh_rest_coeffs(scene.sh_degree);
  std::string header = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(scene.count) + "\n";
  for (const char* p : {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"})
    header += std::string("property float ") + p + "\n";
  for (int i = 0; i < coeffs * 3; ++i) header += "property float f_rest_" + std::to_string(i) + "\n";
  for (const char* p : {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"})
    header += std::string("property float ") + p + "\n";
  header += "end_header\n";
  const size_t per_vertex = 17 + size_t(coeffs) * 3;
  std::vector<float> rows(size_t(scene.count) * per_vertex);
  for (uint32_t i = 0; i < scene.count; ++i) {
    float* r = &rows[size_t(i) * per_vertex];
    size_t k = 0;
    for (int a = 0; a < 3; ++a) r[k++] = scene.positions[size_t(i) * 3 + a];
    for (int a = 0; a < 3; ++a) r[k++] = 0.0f;
    for (int a = 0; a < 3; ++a) r[k++] = scene.sh_dc[size_t(i) * 3 + a];
    for (int c = 0; c < 3; ++c)
      for (int j = 0; j < coeffs; ++j) r[k++] = scene.sh_rest[(size_t(i) * coeffs + j) * 3 + c];
    r[k++] = scene.opacity_logits[i];
    for (int a = 0; a < 3; ++a) r[k++] = scene.log_scales[size_t(i) * 3 + a];
    for (int a = 0; a < 4; ++a) r[k++] = scene.rotations[size_t(i) * 4 + a];
  }
  std::vector<uint8_t> out(header.begin(), header.end());
  const uint8_t* bytes = reinterpret_cast<const uint8_t*>(rows.data());
  out.insert(out.end(), bytes, bytes + rows.size() * sizeof(float));
  return out;
}

void convert_convention(SplatScene& scene, AxisConvention target) {
  if (scene.convention == target) return;
  // Half turn about x, q_x = (0, 1, 0, 0): positions (x, -y, -z); rotations q_x * q; each
  // real SH basis function keeps or flips its sign with its degree in y plus its degree in z.
  static constexpr float kSign[15] = {-1, -1, 1,            // -y, z, -x
                                      -1, 1, 1, -1, 1,      // xy, yz, 2z^2-x^2-y^2, xz, x^2-y^2
                                      -1, 1, -1, -1, 1, -1, 1};
  const int coeffs = sh_rest_coeffs(scene.sh_degree);
  for (uint32_t i = 0; i < scene.count; ++i) {
    scene.positions[size_t(i) * 3 + 1] = -scene.positions[size_t(i) * 3 + 1];
    scene.positions[size_t(i) * 3 + 2] = -scene.positions[size_t(i) * 3 + 2];
    float* q = &scene.rotations[size_t(i) * 4];
    const float w = q[0], x = q[1], y = q[2], z = q[3];
    q[0] = -x;
    q[1] = w;
    q[2] = -z;
    q[3] = y;
    for (int j = 0; j < coeffs; ++j)
      for (int c = 0; c < 3; ++c) scene.sh_rest[(size_t(i) * coeffs + j) * 3 + c] *= kSign[j];
  }
  scene.convention = target;
}

std::vector<uint8_t> read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open " + path);
  return std::vector<uint8_t>(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
}

void write_file(const std::string& path, const std::vector<uint8_t>& bytes) {
  std::ofstream out(path, std::ios::binary);
  if (!out) throw std::runtime_error("cannot write " + path);
  out.write(reinterpret_cast<const char*>(bytes.data()), std::streamsize(bytes.size()));
  if (!out) throw std::runtime_error("failed writing " + path);
}

SplatScene make_random_scene(const RandomSceneOptions& o) {
  std::mt19937_64 rng(o.seed);
  std::normal_distribution<float> normal(0.0f, 1.0f);
  std::uniform_real_distribution<float> uniform(0.0f, 1.0f);
  SplatScene s;
  s.convention = AxisConvention::RUB;
  s.resize(o.count, o.sh_degree);
  const int coeffs = sh_rest_coeffs(o.sh_degree);
  for (uint32_t i = 0; i < o.count; ++i) {
    // Uniform in the ball: a normal direction and radius r u^(1/3).
    float d[3], len2 = 0.0f;
    do {
      len2 = 0.0f;
      for (float& v : d) {
        v = normal(rng);
        len2 += v * v;
      }
    } while (len2 < 1e-12f);
    const float r = o.radius * std::cbrt(uniform(rng)) / std::sqrt(len2);
    for (int k = 0; k < 3; ++k) s.positions[size_t(i) * 3 + k] = d[k] * r;
    for (int k = 0; k < 3; ++k) s.log_scales[size_t(i) * 3 + k] = o.log_scale_mu + o.log_scale_sigma * normal(rng);
    float q[4], ql2 = 0.0f;
    do {
      ql2 = 0.0f;
      for (float& v : q) {
        v = normal(rng);
        ql2 += v * v;
      }
    } while (ql2 < 1e-12f);
    const float inv = 1.0f / std::sqrt(ql2);
    for (int k = 0; k < 4; ++k) s.rotations[size_t(i) * 4 + k] = q[k] * inv;
    s.opacity_logits[i] = normal(rng);
    for (int k = 0; k < 3; ++k)
      s.sh_dc[size_t(i) * 3 + k] = o.sh_degree == 0 ? uniform(rng) : o.sh_sigma * normal(rng);
    for (int j = 0; j < coeffs * 3; ++j) s.sh_rest[size_t(i) * coeffs * 3 + j] = o.sh_sigma * normal(rng);
  }
  return s;
}

}  // namespace gs
