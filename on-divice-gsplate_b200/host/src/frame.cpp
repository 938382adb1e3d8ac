#include "frame.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

namespace gs {

void look_at_c2w_gl(const float eye[3], const float target[3], float c2w[16]) {
  float f[3] = {target[0] - eye[0], target[1] - eye[1], target[2] - eye[2]};
  const float fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (float& v : f) v /= fl;
  // right = forward x up (up = +y), then the true up = right x forward.
  float r[3] = {-f[2], 0.0f, f[0]};
  const float rl = std::sqrt(r[0] * r[0] + r[2] * r[2]);
  for (float& v : r) v /= rl;
  const float u[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
  for (int k = 0; k < 3; ++k) {
    c2w[k * 4 + 0] = r[k];
    c2w[k * 4 + 1] = u[k];
    c2w[k * 4 + 2] = -f[k];
    c2w[k * 4 + 3] = eye[k];
  }
  c2w[12] = c2w[13] = c2w[14] = 0.0f;
  c2w[15] = 1.0f;
}

Camera camera_from_c2w_gl(const float c2w[16], float fx, float fy, float cx, float cy, uint32_t width,
                          uint32_t height) {
  // c2w_cv = c2w_gl diag(1, -1, -1); world -> camera is its transpose.
  Camera cam{};
  for (int r = 0; r < 3; ++r) {
    cam.rotation[0 * 3 + r] = c2w[r * 4 + 0];
    cam.rotation[1 * 3 + r] = -c2w[r * 4 + 1];
    cam.rotation[2 * 3 + r] = -c2w[r * 4 + 2];
    cam.position[r] = c2w[r * 4 + 3];
  }
  for (int r = 0; r < 3; ++r)
    cam.translation[r] = -(cam.rotation[r * 3 + 0] * cam.position[0] + cam.rotation[r * 3 + 1] * cam.position[1] +
                           cam.rotation[r * 3 + 2] * cam.position[2]);
  cam.fx = fx;
  cam.fy = fy;
  cam.cx = cx;
  cam.cy = cy;
  cam.width = width;
  cam.height = height;
  return cam;
}

namespace detail {

void frame_geometry(gs_frame_data& f, const Camera& camera, uint32_t slots, uint32_t sh_stride, int active_degree,
                    uint32_t flags, const float background[3]) {
  std::memset(&f, 0, sizeof(f));
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) f.rot[r][c] = camera.rotation[r * 3 + c];
    f.rot[r][3] = camera.translation[r];
    f.cam_pos[r] = camera.position[r];
  }
  f.intrinsics[0] = camera.fx;
  f.intrinsics[1] = camera.fy;
  f.intrinsics[2] = camera.cx;
  f.intrinsics[3] = camera.cy;
  f.image[0] = camera.width;
  f.image[1] = camera.height;
  f.image[2] = (camera.width + 15u) / 16u;
  f.image[3] = (camera.height + 15u) / 16u;
  f.model[0] = slots;
  f.model[1] = uint32_t(std::max(active_degree, 0));
  f.model[2] = sh_stride;
  f.model[3] = flags;
  for (int c = 0; c < 3; ++c) f.background[c] = background[c];
  f.background[3] = 1.0f / (3.0f * float(camera.width) * float(camera.height));
  f.head[3] = 1.0f;
  f.exposure[0] = f.exposure[1] = f.exposure[2] = 1.0f;
}

void frame_refinement(gs_frame_data& f, const Camera& camera, const HeadRegion& head, float head_weight,
                      const float* gain) {
  for (int c = 0; c < 3; ++c) f.exposure[c] = gain != nullptr && gain[c] > 0.0f ? 1.0f / gain[c] : 1.0f;
  f.head[0] = f.head[1] = f.head[2] = 0.0f;
  f.head[3] = 1.0f;
  if (!head.found) return;
  float t[3];
  for (int r = 0; r < 3; ++r)
    t[r] = camera.rotation[r * 3] * head.center[0] + camera.rotation[r * 3 + 1] * head.center[1] +
           camera.rotation[r * 3 + 2] * head.center[2] + camera.translation[r];
  if (!(t[2] > 0.05f)) return;  // behind (or at) the camera
  f.head[0] = camera.fx * t[0] / t[2] + camera.cx;
  f.head[1] = camera.fy * t[1] / t[2] + camera.cy;
  f.head[2] = camera.fx * head.radius / t[2];
  // Close-ups (the head's radius a quarter of the height or more) keep weight 1.
  f.head[3] = f.head[2] < 0.25f * float(camera.height) ? head_weight : 1.0f;
}

void frame_schedule(gs_frame_data& f, const TrainOptions& o, uint32_t step, float camera_extent, float lambda) {
  constexpr float kBeta1 = 0.9f, kBeta2 = 0.999f, kEpsilon = 1e-15f;  // trainer.cpp:68-70
  const float t = o.iterations > 0 ? std::min(1.0f, float(step) / float(o.iterations)) : 1.0f;
  float lr_pos = o.lr_position;
  if (lr_pos > 0.0f && o.lr_position_final > 0.0f)
    lr_pos = std::exp(std::log(lr_pos) * (1.0f - t) + std::log(o.lr_position_final) * t);
  f.lr0[0] = lr_pos * camera_extent;
  f.lr0[1] = o.lr_scale;
  f.lr0[2] = o.lr_rotation;
  f.lr0[3] = o.lr_opacity;
  f.lr1[0] = o.lr_sh_dc;
  f.lr1[1] = o.lr_sh_rest;
  f.adam[0] = kBeta1;
  f.adam[1] = kBeta2;
  f.adam[2] = kEpsilon;
  const double n = double(step) + 1.0;
  f.bias[0] = float(1.0 / (1.0 - std::pow(double(kBeta1), n)));
  f.bias[1] = float(1.0 / (1.0 - std::pow(double(kBeta2), n)));
  const bool prune_big = o.opacity_reset_interval > 0 && step > o.opacity_reset_interval;
  f.densify0[0] = o.densify_grad_threshold;
  f.densify0[1] = o.percent_dense * camera_extent;
  f.densify0[2] = o.prune_opacity;
  f.densify0[3] = prune_big ? 0.1f * camera_extent : 0.0f;
  f.densify1[0] = prune_big ? 20.0f : 0.0f;
  const uint32_t seed = o.seed * 9781u + step * 6271u;
  std::memcpy(&f.densify1[1], &seed, 4);
  f.densify1[2] = 1.6f;
  f.loss[0] = lambda;
  f.loss[1] = 0.01f * 0.01f;  // SSIM constants for colours in [0, 1]
  f.loss[2] = 0.03f * 0.03f;
}

void pack_params(const SplatScene& scene, int degree, uint32_t sh_stride, std::vector<float>& p,
                 std::vector<float>& sh) {
  p.assign(size_t(scene.count) * 16, 0.0f);
  sh.assign(size_t(scene.count) * sh_stride, 0.0f);
  const int have = sh_rest_coeffs(scene.sh_degree);
  const int use = std::min(have, std::min(sh_rest_coeffs(degree), int(sh_stride / 3)));
  for (uint32_t i = 0; i < scene.count; ++i) {
    float* d = &p[size_t(i) * 16];
    for (int k = 0; k < 3; ++k) {
      d[k] = scene.positions[size_t(i) * 3 + k];
      d[4 + k] = scene.log_scales[size_t(i) * 3 + k];
      d[12 + k] = scene.sh_dc[size_t(i) * 3 + k];
    }
    d[3] = scene.opacity_logits[i];
    d[7] = 1.0f;
    for (int k = 0; k < 4; ++k) d[8 + k] = scene.rotations[size_t(i) * 4 + k];
    for (int j = 0; j < use; ++j)
      for (int c = 0; c < 3; ++c)
        sh[size_t(i) * sh_stride + size_t(j) * 3 + c] = scene.sh_rest[(size_t(i) * have + j) * 3 + c];
  }
}

void check_status(int code, const char* what) {
  if (code != GS_OK) throw std::runtime_error(std::string(what) + ": " + gs_last_error());
}

}  // namespace detail
}  // namespace gs
