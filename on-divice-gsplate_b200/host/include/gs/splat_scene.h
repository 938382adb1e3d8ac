// Gaussian splat scenes on the host and their file formats.
//
// The type and its loaders keep the reference engine's interface
// (engine/include/gs/splat_scene.h): the 3DGS training parameterisation (log scales,
// opacity logits, unnormalised (w, x, y, z) quaternions, SH DC + rest as [coeff][rgb]),
// binary little-endian PLY with the standard 3DGS vertex properties, and the RDF <-> RUB
// axis conversion. Loaders throw std::runtime_error with a message for the user.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace gs {

// Axis convention of a scene's coordinates.
enum class AxisConvention {
  RDF,  // right, down, forward: COLMAP and the standard 3DGS .ply layout
  RUB,  // right, up, back (Y-up worlds: the trainer's datasets, three.js)
};

struct SplatScene {
  uint32_t count = 0;
  int sh_degree = 0;  // 0..3
  bool antialiased = false;
  AxisConvention convention = AxisConvention::RDF;
  std::vector<float> positions;       // 3 per splat
  std::vector<float> log_scales;      // 3 per splat
  std::vector<float> rotations;       // 4 per splat, (w, x, y, z)
  std::vector<float> opacity_logits;  // 1 per splat
  std::vector<float> sh_dc;           // 3 per splat
  std::vector<float> sh_rest;         // sh_rest_coeffs(sh_degree) * 3 per splat, [coeff][rgb]

  void resize(uint32_t n, int degree);
};

// SH coefficients beyond the DC term: 0, 3, 8, 15 for degrees 0..3.
int sh_rest_coeffs(int degree);

struct SceneBounds {
  float center[3];  // per-axis median of the positions
  float radius;     // 90th percentile distance from the center
};
SceneBounds compute_bounds(const SplatScene& scene);

// The vertex element of a binary little-endian PLY, with typed property access. Keeps a
// pointer into the caller's bytes.
class PlyVertices {
 public:
  PlyVertices(const uint8_t* data, size_t size);
  uint64_t count() const { return count_; }
  int find(const std::string& name) const;  // property index, -1 if absent
  float value(uint64_t vertex, int property) const;

 private:
  struct Property {
    std::string name;
    int type;  // index into the scalar type table
    size_t offset;
  };
  const uint8_t* base_ = nullptr;
  uint64_t count_ = 0;
  size_t stride_ = 0;
  std::vector<Property> properties_;
};

SplatScene load_ply(const uint8_t* data, size_t size);
// SPZ v2/v3 (a gzip stream; RUB axes; quantized attributes), as the reference reads it
// (splat_scene.cpp:367-433).
SplatScene load_spz(const uint8_t* data, size_t size);
SplatScene load_splat_file(const uint8_t* data, size_t size);  // PLY or SPZ, detected by magic
std::vector<uint8_t> save_ply(const SplatScene& scene);
// SPZ v3 with `fractional_bits` of position precision (the scene is written in its own
// axes: convert to RUB first for files other SPZ readers open). Not in the reference.
std::vector<uint8_t> save_spz(const SplatScene& scene, int fractional_bits = 12);

// Rewrites the scene in `target` axes (RDF <-> RUB is a half turn about x): positions,
// rotations and the sign of each SH coefficient by its parity in y and z.
void convert_convention(SplatScene& scene, AxisConvention target);

std::vector<uint8_t> read_file(const std::string& path);
void write_file(const std::string& path, const std::vector<uint8_t>& bytes);

// Seeded random scenes with the distributions of the benchmark workloads: means uniform
// in a ball, log-scales N(mu, sigma) per axis, rotations uniform on S^3, opacity logits
// N(0, 1), SH DC U(0, 1) (degree 0) or N(0, sh_sigma) for every coefficient (degree > 0).
// Generator: std::mt19937_64 with std::normal_distribution / uniform_real_distribution.
struct RandomSceneOptions {
  uint32_t count = 0;
  uint64_t seed = 0;
  int sh_degree = 0;
  float radius = 1.0f;
  float log_scale_mu = -4.0f;
  float log_scale_sigma = 0.5f;
  float sh_sigma = 0.2f;
};
SplatScene make_random_scene(const RandomSceneOptions& options);

}  // namespace gs
