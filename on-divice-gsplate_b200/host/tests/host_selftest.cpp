// CPU checks of the host layer, driven by tests/test_host.py:
//   gs_host_selftest scene <dir>   PLY round trip (bit-exact), RDF <-> RUB twice = identity
//   gs_host_selftest frame         one FrameData as 72 hex words (compared with gs_b200.frame)
//   gs_host_selftest camera        look-at camera as 12 floats (rotation rows, translation)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../src/frame.h"
#include "gs/camera.h"
#include "gs/splat_scene.h"
#include "gs/trainer.h"

namespace {

bool same(const gs::SplatScene& a, const gs::SplatScene& b) {
  return a.count == b.count && a.sh_degree == b.sh_degree && a.positions == b.positions &&
         a.log_scales == b.log_scales && a.rotations == b.rotations && a.opacity_logits == b.opacity_logits &&
         a.sh_dc == b.sh_dc && a.sh_rest == b.sh_rest;
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

}  // namespace

int main(int argc, char** argv) {
  try {
    const std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "scene" && argc > 2) return scene_checks(argv[2]);
    if (mode == "frame") return frame_words();
    if (mode == "camera") return camera_floats();
    std::fprintf(stderr, "usage: %s scene <dir> | frame | camera\n", argv[0]);
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
