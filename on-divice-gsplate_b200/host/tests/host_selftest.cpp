// CPU checks of the host layer, driven by tests/test_host.py:
//   gs_host_selftest scene <dir>   PLY round trip (bit-exact), RDF <-> RUB twice = identity,
//                                  SPZ v3 and v2 round trips within their quantization
//   gs_host_selftest frame         one FrameData as 72 hex words (compared with gs_b200.frame)
//   gs_host_selftest camera        look-at camera as 12 floats (rotation rows, translation)
//   gs_host_selftest dataset <dir> <width> <max_init>
//                                  load_dataset + initialize_gaussians: a JSON summary on
//                                  stdout, frame 0's RGBA in <dir>/frame0.rgba
//   gs_host_selftest head <xyz> <ux> <uy> <uz> <weight>
//                                  estimate_head over the float32 xyz triples in <xyz> with
//                                  world up (ux, uy, uz), then the head and exposure words of
//                                  a FrameData for the test camera with gains (0.8, 1, 1.25)
//   gs_host_selftest refine        the pose, exposure and motion-rig arithmetic of the
//                                  trainer's corrections (rotations, rigid corrections, Adam,
//                                  capture-order blends, centred gains, node placement and
//                                  the rig energies' gradients against central differences)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <zlib.h>

#include "../src/frame.h"
#include "../src/node_rig.h"
#include "../src/refinement.h"
#include "gs/camera.h"
#include "gs/dataset.h"
#include "gs/splat_scene.h"
#include "gs/trainer.h"

namespace {

bool same(const gs::SplatScene& a, const gs::SplatScene& b) {
  return a.count == b.count && a.sh_degree == b.sh_degree && a.positions == b.positions &&
         a.log_scales == b.log_scales && a.rotations == b.rotations && a.opacity_logits == b.opacity_logits &&
         a.sh_dc == b.sh_dc && a.sh_rest == b.sh_rest;
}

void expect(bool ok, const std::string& what) {
  if (!ok) throw std::runtime_error(what);
}

// The SPZ quantization steps: 2^-12 in position (12 fractional bits), 1/255 of colour
// (DC / 0.15), 1/16 of log scale, 1/255 of alpha, 1/128 of SH; the rotation to 9 bits.
void check_spz(const gs::SplatScene& s, const gs::SplatScene& back, const char* what) {
  expect(back.count == s.count && back.sh_degree == s.sh_degree, std::string(what) + ": count/degree");
  for (uint32_t i = 0; i < s.count; ++i) {
    for (int k = 0; k < 3; ++k) {
      const size_t a = size_t(i) * 3 + k;
      expect(std::fabs(back.positions[a] - s.positions[a]) <= 0.5f / 4096.0f + 1e-6f, std::string(what) + ": position");
      expect(std::fabs(back.log_scales[a] - s.log_scales[a]) <= 1.0f / 32.0f + 1e-5f, std::string(what) + ": scale");
      expect(std::fabs(back.sh_dc[a] - s.sh_dc[a]) <= 0.5f / 255.0f / 0.15f + 1e-5f, std::string(what) + ": colour");
    }
    const float o0 = 1.0f / (1.0f + std::exp(-s.opacity_logits[i])), o1 = 1.0f / (1.0f + std::exp(-back.opacity_logits[i]));
    expect(std::fabs(o0 - o1) <= 0.5f / 255.0f + 1e-5f, std::string(what) + ": opacity");
    const float* q0 = &s.rotations[size_t(i) * 4];
    const float* q1 = &back.rotations[size_t(i) * 4];
    const float n0 = std::sqrt(q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3]);
    const float dot = (q0[0] * q1[0] + q0[1] * q1[1] + q0[2] * q1[2] + q0[3] * q1[3]) / n0;
    expect(std::fabs(dot) >= 0.9999f, std::string(what) + ": rotation");  // the same rotation (q or -q)
    const int c = gs::sh_rest_coeffs(s.sh_degree);
    for (int j = 0; j < c * 3; ++j) {
      const size_t a = size_t(i) * c * 3 + j;
      const float v = std::min(std::max(s.sh_rest[a], -1.0f), 127.0f / 128.0f);
      expect(std::fabs(back.sh_rest[a] - v) <= 0.5f / 128.0f + 1e-6f, std::string(what) + ": sh");
    }
  }
}

// A v2 file (3-byte rotations) written byte by byte from the published layout.
std::vector<uint8_t> spz_v2(const gs::SplatScene& s) {
  const uint32_t n = s.count;
  const int coeffs = gs::sh_rest_coeffs(s.sh_degree);
  std::vector<uint8_t> raw(16);
  const uint32_t head[3] = {0x5053474eu, 2u, n};
  std::memcpy(raw.data(), head, 12);
  raw[12] = uint8_t(s.sh_degree);
  raw[13] = 12;
  auto q8 = [](float v) { return uint8_t(std::lround(std::min(std::max(v, 0.0f), 255.0f))); };
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      const uint32_t u = uint32_t(std::lround(s.positions[size_t(i) * 3 + k] * 4096.0f)) & 0xffffffu;
      raw.insert(raw.end(), {uint8_t(u), uint8_t(u >> 8), uint8_t(u >> 16)});
    }
  for (uint32_t i = 0; i < n; ++i) raw.push_back(q8(255.0f / (1.0f + std::exp(-s.opacity_logits[i]))));
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) raw.push_back(q8((s.sh_dc[size_t(i) * 3 + k] * 0.15f + 0.5f) * 255.0f));
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) raw.push_back(q8((s.log_scales[size_t(i) * 3 + k] + 10.0f) * 16.0f));
  for (uint32_t i = 0; i < n; ++i) {
    const float* q = &s.rotations[size_t(i) * 4];
    const float len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const float sign = q[0] < 0.0f ? -1.0f : 1.0f;  // w >= 0
    for (int k = 1; k <= 3; ++k) raw.push_back(q8((sign * q[k] / len + 1.0f) * 127.5f));
  }
  for (uint32_t i = 0; i < n; ++i)
    for (int j = 0; j < coeffs * 3; ++j) raw.push_back(q8(s.sh_rest[size_t(i) * coeffs * 3 + j] * 128.0f + 128.0f));
  std::vector<uint8_t> out(compressBound(uLong(raw.size())) + 64);
  z_stream zs{};
  deflateInit2(&zs, Z_BEST_SPEED, Z_DEFLATED, 16 + MAX_WBITS, 8, Z_DEFAULT_STRATEGY);
  zs.next_in = raw.data();
  zs.avail_in = uInt(raw.size());
  zs.next_out = out.data();
  zs.avail_out = uInt(out.size());
  deflate(&zs, Z_FINISH);
  out.resize(out.size() - zs.avail_out);
  deflateEnd(&zs);
  return out;
}

int scene_checks(const std::string& dir) {
  for (int degree = 0; degree <= 3; ++degree) {
    gs::RandomSceneOptions o;
    o.count = 1000;
    o.seed = 11 + uint64_t(degree);
    o.sh_degree = degree;
    const gs::SplatScene s = gs::make_random_scene(o);
    const std::string path = dir + "/scene_" + std::to_string(degree) + ".ply";
    gs::write_file(path, gs::save_ply(s));
    const std::vector<uint8_t> bytes = gs::read_file(path);
    const gs::SplatScene back = gs::load_splat_file(bytes.data(), bytes.size());
    if (!same(s, back)) throw std::runtime_error("PLY round trip differs at degree " + std::to_string(degree));
    gs::SplatScene turned = back;
    turned.convention = gs::AxisConvention::RUB;
    gs::convert_convention(turned, gs::AxisConvention::RDF);
    gs::convert_convention(turned, gs::AxisConvention::RUB);
    gs::SplatScene q = turned;
    // Twice a half turn: positions and SH back exactly, the quaternion negated (the same rotation).
    for (float& v : q.rotations) v = -v;
    if (q.positions != s.positions || q.sh_rest != s.sh_rest || q.rotations != s.rotations)
      throw std::runtime_error("convention round trip is not the identity at degree " + std::to_string(degree));
    const std::vector<uint8_t> spz = gs::save_spz(s, 12);
    check_spz(s, gs::load_splat_file(spz.data(), spz.size()), "spz v3");
    const std::vector<uint8_t> v2 = spz_v2(s);
    gs::SplatScene b2 = gs::load_splat_file(v2.data(), v2.size());
    // v2 rotations keep 8 bits per component: compare to a looser bound.
    for (uint32_t i = 0; i < s.count; ++i) {
      const float* q0 = &s.rotations[size_t(i) * 4];
      const float* q1 = &b2.rotations[size_t(i) * 4];
      const float n0 = std::sqrt(q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3]);
      expect(std::fabs(q0[0] * q1[0] + q0[1] * q1[1] + q0[2] * q1[2] + q0[3] * q1[3]) / n0 >= 0.995f, "spz v2: rotation");
      for (int k = 0; k < 4; ++k) b2.rotations[size_t(i) * 4 + k] = q0[k];
    }
    check_spz(s, b2, "spz v2");
  }
  std::printf("ok\n");
  return 0;
}

gs::Camera test_camera() {
  const float eye[3] = {0.0f, 0.0f, 3.0f}, target[3] = {0.0f, 0.0f, 0.0f};
  float c2w[16];
  gs::look_at_c2w_gl(eye, target, c2w);
  return gs::camera_from_c2w_gl(c2w, 500.0f, 500.0f, 180.0f, 320.0f, 360, 640);
}

int frame_words() {
  const gs::Camera cam = test_camera();
  const gs::TrainOptions o;
  gs_frame_data f;
  const float bg[3] = {0.1f, 0.2f, 0.3f};
  const uint32_t step = 10;
  const float t = std::min(1.0f, float(step) / float(o.iterations - 1));
  const float lambda = o.lambda_dssim + (o.lambda_dssim_end - o.lambda_dssim) * t;
  gs::detail::frame_geometry(f, cam, 20000, 45, int(std::min<uint32_t>(3, step / o.sh_degree_interval)),
                             GS_FLAG_SSIM, bg);
  gs::detail::frame_schedule(f, o, step, 3.3f, lambda);
  uint32_t w[72];
  std::memcpy(w, &f, sizeof(w));
  for (int k = 0; k < 72; ++k) std::printf("%08x%c", w[k], k == 71 ? '\n' : ' ');
  return 0;
}

int camera_floats() {
  const gs::Camera c = test_camera();
  for (int k = 0; k < 9; ++k) std::printf("%.9g ", c.rotation[k]);
  std::printf("%.9g %.9g %.9g\n", c.translation[0], c.translation[1], c.translation[2]);
  return 0;
}

int dataset_summary(const std::string& dir, uint32_t width, uint32_t max_init) {
  const gs::Dataset ds = gs::load_dataset(dir, width);
  gs::InitOptions io;
  io.max_gaussians = max_init;
  gs::InitStats st;
  const gs::SplatScene init = gs::initialize_gaussians(ds, io, &st);
  gs::write_file(dir + "/frame0.rgba", ds.frames.at(0).rgba);
  // The initial gaussians' positions and log-scales (float32) for the caller to check.
  std::vector<uint8_t> bytes(init.positions.size() * 4), scales(init.log_scales.size() * 4);
  std::memcpy(bytes.data(), init.positions.data(), bytes.size());
  std::memcpy(scales.data(), init.log_scales.data(), scales.size());
  gs::write_file(dir + "/init.xyz", bytes);
  gs::write_file(dir + "/init.logscale", scales);
  float smin = INFINITY, smax = -INFINITY;
  for (float v : init.log_scales) {
    smin = std::min(smin, v);
    smax = std::max(smax, v);
  }
  std::printf("{\"name\": \"%s\", \"width\": %u, \"height\": %u, \"fx\": %.6g, \"fy\": %.6g, \"cx\": %.6g, "
              "\"cy\": %.6g, \"frames\": %zu, \"holdout\": %zu, \"skipped\": %zu, \"has_masks\": %s, \"has_depth\": %s, "
              "\"points\": %zu, "
              "\"extent\": %.6g, \"names\": [",
              ds.name.c_str(), ds.width, ds.height, ds.fx, ds.fy, ds.cx, ds.cy, ds.frames.size(), ds.holdout_count(),
              ds.skipped.size(), ds.has_masks ? "true" : "false", ds.has_depth ? "true" : "false", ds.points.size() / 3,
              ds.camera_extent);
  for (size_t i = 0; i < ds.frames.size(); ++i)
    std::printf("%s\"%s\"", i ? ", " : "", ds.frames[i].name.c_str());
  std::printf("], \"skipped_why\": [");
  for (size_t i = 0; i < ds.skipped.size(); ++i) {
    std::string why = ds.skipped[i];
    for (char& ch : why)
      if (ch == '"' || ch == '\\') ch = '\'';
    std::printf("%s\"%s\"", i ? ", " : "", why.c_str());
  }
  std::printf("], \"init_source\": \"%s\", \"init_raw\": %zu, \"init_count\": %u, \"init_voxel\": %.6g, "
              "\"log_scale_min\": %.6g, \"log_scale_max\": %.6g, \"init_opacity_logit\": %.6g}\n",
              st.source.c_str(), st.raw_points, init.count, st.voxel_size, smin, smax,
              init.count ? init.opacity_logits[0] : 0.0f);
  return 0;
}

int head_summary(const std::string& path, const float up[3], float weight) {
  const std::vector<uint8_t> bytes = gs::read_file(path);
  gs::SplatScene s;
  s.resize(uint32_t(bytes.size() / 12), 0);
  std::memcpy(s.positions.data(), bytes.data(), size_t(s.count) * 12);
  const gs::HeadRegion h = gs::estimate_head(s, up);
  gs_frame_data f;
  const float bg[3] = {0.0f, 0.0f, 0.0f}, gain[3] = {0.8f, 1.0f, 1.25f};
  const gs::Camera cam = test_camera();
  gs::detail::frame_geometry(f, cam, s.count, 0, 0, 0u, bg);
  gs::detail::frame_refinement(f, cam, h, weight, gain);
  std::printf("{\"found\": %s, \"center\": [%.9g, %.9g, %.9g], \"radius\": %.9g, \"height\": %.9g, "
              "\"frame_head\": [%.9g, %.9g, %.9g, %.9g], \"frame_exposure\": [%.9g, %.9g, %.9g]}\n",
              h.found ? "true" : "false", h.center[0], h.center[1], h.center[2], h.radius, h.subject_height,
              f.head[0], f.head[1], f.head[2], f.head[3], f.exposure[0], f.exposure[1], f.exposure[2]);
  return 0;
}

int refine_checks() {
  using namespace gs::refine;
  std::mt19937 rng(12);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  auto close = [](double a, double b, double tol) { return std::fabs(a - b) <= tol; };
  double worst = 0.0;
  // Rotations: exp/log round trip, composition against matrices, slerp end points and middle.
  for (int trial = 0; trial < 200; ++trial) {
    const Vec3 w{1.5 * u(rng), 1.5 * u(rng), 1.5 * u(rng)};
    const Vec3 back = Rotation::exp(w).log();
    for (int c = 0; c < 3; ++c) worst = std::max(worst, std::fabs(back[c] - w[c]));
    const Rotation a = Rotation::exp(w), b = Rotation::exp({u(rng), u(rng), u(rng)});
    double A[9], B[9], AB[9];
    a.to_matrix(A);
    b.to_matrix(B);
    a.after(b).to_matrix(AB);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double v = 0.0;
        for (int k = 0; k < 3; ++k) v += A[r * 3 + k] * B[k * 3 + c];
        worst = std::max(worst, std::fabs(v - AB[r * 3 + c]));
      }
    const Rotation s0 = Rotation::slerp(a, b, 0.0), s1 = Rotation::slerp(a, b, 1.0);
    const Rotation mid = Rotation::slerp(a, b, 0.5);
    expect(close(s0.after(Rotation{{a.q[0], -a.q[1], -a.q[2], -a.q[3]}}).degrees(), 0.0, 1e-6), "slerp at 0");
    expect(close(s1.after(Rotation{{b.q[0], -b.q[1], -b.q[2], -b.q[3]}}).degrees(), 0.0, 1e-6), "slerp at 1");
    const double ab = b.after(Rotation{{a.q[0], -a.q[1], -a.q[2], -a.q[3]}}).degrees();
    const double am = mid.after(Rotation{{a.q[0], -a.q[1], -a.q[2], -a.q[3]}}).degrees();
    expect(close(am, 0.5 * ab, 1e-6), "slerp halfway");
  }
  expect(worst < 1e-9, "rotation round trips: " + std::to_string(worst));
  // A correction followed by a step equals the camera composed by hand.
  {
    gs::Camera cam = gs::camera_from_c2w_gl(std::array<float, 16>{0.8f, 0.0f, 0.6f, 1.0f, 0.0f, 1.0f, 0.0f, 0.5f,
                                                                  -0.6f, 0.0f, 0.8f, 2.0f, 0, 0, 0, 1}
                                                .data(),
                                            100.0f, 100.0f, 32.0f, 24.0f, 64, 48);
    RigidFix fix;
    fix = fix.then({0.01, -0.02, 0.03}, {0.02, 0.01, -0.03});
    fix = fix.then({-0.005, 0.0, 0.01}, {0.0, 0.04, 0.0});
    const gs::Camera got = fix.apply(cam);
    double U[9];
    fix.turn.to_matrix(U);
    for (int r = 0; r < 3; ++r) {
      double t = fix.shift[r];
      for (int c = 0; c < 3; ++c) {
        double v = 0.0;
        for (int k = 0; k < 3; ++k) v += U[r * 3 + k] * cam.rotation[k * 3 + c];
        expect(close(v, got.rotation[r * 3 + c], 1e-6), "corrected rotation");
        t += U[r * 3 + c] * cam.translation[c];
      }
      expect(close(t, got.translation[r], 1e-6), "corrected translation");
    }
    for (int c = 0; c < 3; ++c) {
      double p = 0.0;
      for (int r = 0; r < 3; ++r) p -= double(got.rotation[r * 3 + c]) * got.translation[r];
      expect(close(p, got.position[c], 1e-5), "corrected centre");
    }
  }
  // Adam's first step is the rate against the gradient's sign.
  {
    Adam<6> adam;
    const std::array<double, 6> step = adam.step({3.0, -1e-8, 0.0, 2.0, -5.0, 1e3}, {1, 2, 3, 4, 5, 6});
    const double want[6] = {-1.0, 2.0, 0.0, -4.0, 5.0, -6.0};
    for (int i = 0; i < 6; ++i) expect(close(step[i], want[i], 1e-9), "Adam first step");
  }
  // Capture order: the nearest usable trained frames on either side, never the frame itself.
  CaptureOrder order;
  order.build(10, {1, 3, 4, 7});
  auto all = [](size_t) { return true; };
  CaptureOrder::Span s = order.around(5, all);
  expect(s.lo == 4 && s.hi == 7 && close(s.t, 1.0 / 3.0, 1e-12), "span of 5");
  s = order.around(0, all);
  expect(s.lo == CaptureOrder::kNone && s.hi == 1 && s.t == 1.0, "span of 0");
  s = order.around(9, all);
  expect(s.lo == 7 && s.hi == CaptureOrder::kNone && s.t == 0.0, "span of 9");
  s = order.around(3, all);
  expect(s.lo == 1 && s.hi == 4, "span of a trained frame");
  s = order.around(5, [](size_t f) { return f != 4; });
  expect(s.lo == 3 && s.hi == 7, "span skipping an unusable frame");
  // Gains: centred on the measured trained views, blended for the others.
  {
    GainTable g;
    g.reset(10);
    const double f1[8] = {1000, 1000, 1000, 600, 2000, 1000, 500, 0};  // gains 2, 1, 0.5
    const double f3[8] = {1000, 1000, 1000, 600, 1000, 1000, 1000, 0};  // gains 1, 1, 1
    g.observe(1, f1, 0.3);
    g.observe(3, f3, 0.3);
    const double few[8] = {1000, 1000, 1000, 10, 9000, 9000, 9000, 0};  // too few pixels: ignored
    g.observe(3, few, 0.3);
    const std::array<float, 3> a = g.gains(1, order), b = g.gains(3, order), m = g.gains(2, order);
    expect(close(a[0], std::sqrt(2.0), 1e-5) && close(a[1], 1.0, 1e-6) && close(a[2], std::sqrt(0.5), 1e-5),
           "centred gains of frame 1");
    expect(close(double(a[0]) * b[0], 1.0, 1e-5) && close(double(a[2]) * b[2], 1.0, 1e-5), "centred gains of frame 3");
    expect(close(m[0], 1.0, 1e-5), "frame 2 halfway between 1 and 3 in log gain");
    const GainTable::Spread spread = g.spread(order);
    expect(spread.updates == 2 && spread.low <= spread.high, "gain spread");
  }
  // The rig: placement, and its energies' gradients against central differences.
  double grad_err = 0.0;
  {
    std::vector<float> xyz;
    std::normal_distribution<float> n(0.0f, 0.3f);
    for (int i = 0; i < 6000; ++i) {
      const float cx = i % 2 ? 1.0f : -1.0f;
      xyz.insert(xyz.end(), {cx + n(rng), n(rng), 0.5f * n(rng)});
    }
    NodeRig rig;
    rig.place(xyz, 24, 10, 0.1f);
    expect(rig.size() == 24 && rig.spacing() > 0.0f, "rig size");
    for (const NodeRig::Node& node : rig.nodes()) expect(node.radius > 0.0f, "node radius");
    for (size_t f : {1, 3, 7})
      for (size_t k = 0; k < rig.size(); ++k)
        rig.set(f, k, {0.05 * u(rng), 0.05 * u(rng), 0.05 * u(rng)}, {0.02 * u(rng), 0.02 * u(rng), 0.02 * u(rng)});
    RigEnergy w;
    w.decay = 0.3;
    w.rigidity = 0.7;
    w.smoothness = 0.2;
    w.centring = 0.4;
    // Frame 4: shifts anywhere, turns at zero (where a turn applied on top of the node's and
    // the rotation vector agree to first order).
    for (size_t k = 0; k < rig.size(); ++k) rig.set(4, k, {0.0, 0.0, 0.0}, {0.03 * u(rng), 0.03 * u(rng), 0.03 * u(rng)});
    const std::vector<double> grad = rig.energy_gradient(4, w, order);
    double scale = 0.0;
    for (double v : grad) scale = std::max(scale, std::fabs(v));
    const double h = 1e-6;
    for (size_t k = 0; k < rig.size(); ++k)
      for (int part = 0; part < 2; ++part)
        for (int c = 0; c < 3; ++c) {
          NodeMotion m = rig.pose(4)[k];
          Vec3& x = part == 0 ? m.shift : m.turn;
          const double saved = x[c];
          x[c] = saved + h;
          rig.set(4, k, m.turn, m.shift);
          const double up = rig.energy(4, w, order);
          x[c] = saved - h;
          rig.set(4, k, m.turn, m.shift);
          const double down = rig.energy(4, w, order);
          x[c] = saved;
          rig.set(4, k, m.turn, m.shift);
          grad_err = std::max(grad_err, std::fabs((up - down) / (2.0 * h) - grad[k * 6 + part * 3 + c]) / scale);
        }
    const std::vector<float> table = rig.table(rig.pose(4));
    expect(table.size() == rig.size() * 20, "node table size");
  }
  expect(grad_err < 1e-5, "rig energy gradient vs central differences: " + std::to_string(grad_err));
  std::printf("{\"rotation_err\": %.3g, \"rig_gradient_err\": %.3g}\n", worst, grad_err);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    const std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "scene" && argc > 2) return scene_checks(argv[2]);
    if (mode == "frame") return frame_words();
    if (mode == "refine") return refine_checks();
    if (mode == "camera") return camera_floats();
    if (mode == "dataset" && argc > 4) return dataset_summary(argv[2], uint32_t(std::atoi(argv[3])), uint32_t(std::atoi(argv[4])));
    if (mode == "head" && argc > 6) {
      const float up[3] = {float(std::atof(argv[3])), float(std::atof(argv[4])), float(std::atof(argv[5]))};
      return head_summary(argv[2], up, float(std::atof(argv[6])));
    }
    std::fprintf(stderr, "usage: %s scene <dir> | frame | camera\n", argv[0]);
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
