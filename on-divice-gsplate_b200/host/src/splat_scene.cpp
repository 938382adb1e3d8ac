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

#include <zlib.h>

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

// ---- SPZ ----
// Layout (v2/v3): a gzip stream holding a 16-byte header -- magic "NGSP" (0x5053474e LE),
// version, point count (u32 each), SH degree, fractional bits, flags (bit 0: antialiased),
// reserved (u8 each) -- then per-attribute blocks over all points: positions (3 x 24-bit
// signed fixed point), alpha (u8, sigmoid(opacity) x 255), colour (3 x u8, DC x 0.15 + 0.5
// in [0, 1]), log-scales (3 x u8, (s + 10) x 16), rotations (v2: 3 x u8 of x, y, z in
// [-1, 1] with w >= 0; v3: u32 "smallest three": the largest component's index in the top
// 2 bits, the other three as 9-bit magnitudes / sqrt(2) with a sign bit, last component
// lowest) and SH beyond DC (coefficients x rgb, u8 around 128, / 128).
namespace {

constexpr uint32_t kSpzMagic = 0x5053474eu;
constexpr float kSpzColourScale = 0.15f;

std::vector<uint8_t> gunzip(const uint8_t* data, size_t size) {
  z_stream zs{};
  if (inflateInit2(&zs, 16 + MAX_WBITS) != Z_OK) throw std::runtime_error("SPZ: zlib init failed");
  std::vector<uint8_t> out;
  zs.next_in = const_cast<Bytef*>(data);
  zs.avail_in = uInt(size);
  int rc = Z_OK;
  do {
    const size_t at = out.size();
    out.resize(at + std::max<size_t>(size * 4, 1 << 16));
    zs.next_out = out.data() + at;
    zs.avail_out = uInt(out.size() - at);
    rc = inflate(&zs, Z_NO_FLUSH);
    out.resize(out.size() - zs.avail_out);
    if (rc != Z_OK && rc != Z_STREAM_END) {
      inflateEnd(&zs);
      throw std::runtime_error("SPZ: not a valid gzip stream");
    }
  } while (rc != Z_STREAM_END && (zs.avail_in > 0 || zs.avail_out == 0));
  inflateEnd(&zs);
  if (rc != Z_STREAM_END) throw std::runtime_error("SPZ: gzip stream is truncated");
  return out;
}

std::vector<uint8_t> gzip(const std::vector<uint8_t>& raw) {
  z_stream zs{};
  if (deflateInit2(&zs, Z_BEST_SPEED, Z_DEFLATED, 16 + MAX_WBITS, 8, Z_DEFAULT_STRATEGY) != Z_OK)
    throw std::runtime_error("SPZ: zlib init failed");
  std::vector<uint8_t> out(deflateBound(&zs, uLong(raw.size())) + 64);
  zs.next_in = const_cast<Bytef*>(raw.data());
  zs.avail_in = uInt(raw.size());
  zs.next_out = out.data();
  zs.avail_out = uInt(out.size());
  const int rc = deflate(&zs, Z_FINISH);
  out.resize(out.size() - zs.avail_out);
  deflateEnd(&zs);
  if (rc != Z_STREAM_END) throw std::runtime_error("SPZ: compression failed");
  return out;
}

uint8_t quantize(float v) { return uint8_t(std::lround(std::min(std::max(v, 0.0f), 255.0f))); }

}  // namespace

SplatScene load_spz(const uint8_t* data, size_t size) {
  if (size >= 4 && load_le<uint32_t>(data) == kSpzMagic)
    throw std::runtime_error("SPZ: uncompressed (v4) files are not supported (v2/v3 only)");
  if (size < 2 || data[0] != 0x1f || data[1] != 0x8b) throw std::runtime_error("not an SPZ file");
  const std::vector<uint8_t> raw = gunzip(data, size);
  if (raw.size() < 16 || load_le<uint32_t>(raw.data()) != kSpzMagic) throw std::runtime_error("SPZ: bad header");
  const uint32_t version = load_le<uint32_t>(raw.data() + 4), n = load_le<uint32_t>(raw.data() + 8);
  const int file_degree = raw[12], fractional_bits = raw[13];
  if (version < 2 || version > 3) throw std::runtime_error("SPZ: version " + std::to_string(version) + " (v2/v3 only)");
  if (file_degree > 4) throw std::runtime_error("SPZ: bad SH degree");
  const int file_coeffs = file_degree == 4 ? 24 : sh_rest_coeffs(file_degree);
  const int degree = std::min(file_degree, 3), coeffs = sh_rest_coeffs(degree);
  const size_t rot_bytes = version >= 3 ? 4 : 3;
  const size_t positions = 16, alphas = positions + size_t(n) * 9, colours = alphas + n, scales = colours + size_t(n) * 3,
               rotations = scales + size_t(n) * 3, sh = rotations + size_t(n) * rot_bytes,
               end = sh + size_t(n) * file_coeffs * 3;
  if (n == 0 || raw.size() < end) throw std::runtime_error("SPZ: data is truncated");
  SplatScene s;
  s.convention = AxisConvention::RUB;
  s.antialiased = (raw[14] & 1u) != 0;
  s.resize(n, degree);
  const float unit = 1.0f / float(1u << fractional_bits);
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      const uint8_t* p = &raw[positions + (size_t(i) * 3 + k) * 3];
      int32_t v = int32_t(uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16);
      if (v & 0x800000) v -= 0x1000000;  // sign of the 24-bit value
      s.positions[size_t(i) * 3 + k] = float(v) * unit;
      s.sh_dc[size_t(i) * 3 + k] = (float(raw[colours + size_t(i) * 3 + k]) / 255.0f - 0.5f) / kSpzColourScale;
      s.log_scales[size_t(i) * 3 + k] = float(raw[scales + size_t(i) * 3 + k]) / 16.0f - 10.0f;
    }
    const float a = std::min(std::max(float(raw[alphas + i]) / 255.0f, 1e-6f), 1.0f - 1e-6f);
    s.opacity_logits[i] = std::log(a / (1.0f - a));
    float xyzw[4];
    const uint8_t* r = &raw[rotations + size_t(i) * rot_bytes];
    if (version >= 3) {
      uint32_t bits = load_le<uint32_t>(r);
      const int largest = int(bits >> 30);
      float sum = 0.0f;
      for (int c = 3; c >= 0; --c) {
        if (c == largest) continue;
        const float mag = float(bits & 511u) / 511.0f * 0.70710678118654752f;
        xyzw[c] = (bits >> 9) & 1u ? -mag : mag;
        sum += xyzw[c] * xyzw[c];
        bits >>= 10;
      }
      xyzw[largest] = std::sqrt(std::max(0.0f, 1.0f - sum));
    } else {
      for (int k = 0; k < 3; ++k) xyzw[k] = float(r[k]) / 127.5f - 1.0f;
      xyzw[3] = std::sqrt(std::max(0.0f, 1.0f - (xyzw[0] * xyzw[0] + xyzw[1] * xyzw[1] + xyzw[2] * xyzw[2])));
    }
    s.rotations[size_t(i) * 4 + 0] = xyzw[3];  // (w, x, y, z)
    for (int k = 0; k < 3; ++k) s.rotations[size_t(i) * 4 + 1 + k] = xyzw[k];
    for (int j = 0; j < coeffs; ++j)
      for (int c = 0; c < 3; ++c)
        s.sh_rest[(size_t(i) * coeffs + j) * 3 + c] =
            (float(raw[sh + (size_t(i) * file_coeffs + j) * 3 + c]) - 128.0f) / 128.0f;
  }
  return s;
}

std::vector<uint8_t> save_spz(const SplatScene& s, int fractional_bits) {
  if (fractional_bits < 0 || fractional_bits > 23) throw std::runtime_error("save_spz: fractional_bits 0..23");
  const uint32_t n = s.count;
  const int coeffs = sh_rest_coeffs(s.sh_degree);
  std::vector<uint8_t> raw(16 + size_t(n) * (9 + 1 + 3 + 3 + 4 + size_t(coeffs) * 3));
  const uint32_t head[3] = {kSpzMagic, 3u, n};
  std::memcpy(raw.data(), head, 12);
  raw[12] = uint8_t(s.sh_degree);
  raw[13] = uint8_t(fractional_bits);
  raw[14] = s.antialiased ? 1u : 0u;
  const size_t positions = 16, alphas = positions + size_t(n) * 9, colours = alphas + n, scales = colours + size_t(n) * 3,
               rotations = scales + size_t(n) * 3, sh = rotations + size_t(n) * 4;
  const float unit = float(1u << fractional_bits);
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      const long v = std::min(std::max(std::lround(s.positions[size_t(i) * 3 + k] * unit), -0x800000l), 0x7fffffl);
      const uint32_t u = uint32_t(v) & 0xffffffu;
      uint8_t* p = &raw[positions + (size_t(i) * 3 + k) * 3];
      p[0] = uint8_t(u);
      p[1] = uint8_t(u >> 8);
      p[2] = uint8_t(u >> 16);
      raw[colours + size_t(i) * 3 + k] = quantize((s.sh_dc[size_t(i) * 3 + k] * kSpzColourScale + 0.5f) * 255.0f);
      raw[scales + size_t(i) * 3 + k] = quantize((s.log_scales[size_t(i) * 3 + k] + 10.0f) * 16.0f);
    }
    raw[alphas + i] = quantize(255.0f / (1.0f + std::exp(-s.opacity_logits[i])));
    // (x, y, z, w), normalised, the largest component made positive.
    const float* q = &s.rotations[size_t(i) * 4];
    float xyzw[4] = {q[1], q[2], q[3], q[0]};
    const float len = std::sqrt(xyzw[0] * xyzw[0] + xyzw[1] * xyzw[1] + xyzw[2] * xyzw[2] + xyzw[3] * xyzw[3]);
    int largest = 0;
    for (int c = 0; c < 4; ++c) {
      xyzw[c] = len > 0.0f ? xyzw[c] / len : (c == 3 ? 1.0f : 0.0f);
      if (std::fabs(xyzw[c]) > std::fabs(xyzw[largest])) largest = c;
    }
    const float flip = xyzw[largest] < 0.0f ? -1.0f : 1.0f;
    uint32_t bits = uint32_t(largest) << 30;
    int shift = 20;
    for (int c = 0; c < 4; ++c) {
      if (c == largest) continue;
      const float v = xyzw[c] * flip;
      const uint32_t mag = uint32_t(std::min(511l, std::lround(std::fabs(v) * 1.41421356237309505f * 511.0f)));
      bits |= ((v < 0.0f ? 1u : 0u) << 9 | mag) << shift;
      shift -= 10;
    }
    std::memcpy(&raw[rotations + size_t(i) * 4], &bits, 4);
    for (int j = 0; j < coeffs * 3; ++j)
      raw[sh + size_t(i) * coeffs * 3 + j] = quantize(s.sh_rest[size_t(i) * coeffs * 3 + j] * 128.0f + 128.0f);
  }
  return gzip(raw);
}

SplatScene load_splat_file(const uint8_t* data, size_t size) {
  if (size >= 3 && std::memcmp(data, "ply", 3) == 0) return load_ply(data, size);
  if (size >= 4 && ((data[0] == 0x1f && data[1] == 0x8b) || load_le<uint32_t>(data) == kSpzMagic))
    return load_spz(data, size);
  throw std::runtime_error("not a PLY or SPZ splat file");
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
