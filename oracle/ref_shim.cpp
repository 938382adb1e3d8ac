// Test infrastructure only: the glue that builds oracle/_ref/libgs_ref.so, the reference's
// own FP64 CPU forward + loss, so the oracle's restatement can be checked against it.
//
// The reference's only CPU code for the training step is the FP64 projection, per-pixel
// compositing and L1 + SSIM loss of engine/src/train_selftest.cpp:27-283 (`project`,
// `reference_ssim`, `reference_loss`). That file cannot be compiled whole outside the engine:
// its header pulls gs/trainer.h -> gs/vk_context.h -> <vulkan/vulkan.h>, and the rest of the
// file needs generated SPIR-V headers. The lines the CPU maths occupies depend only on
// gs::Camera (engine/include/gs/camera.h:10-16) and the standard library, so oracle/Makefile's
// `ref` target copies that line range from the reference checkout into oracle/_ref/ (never
// into the repository) and this file compiles it with a Camera of the same fields. Only
// tests/ load the result.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace gs {

// The fields of gs::Camera (engine/include/gs/camera.h:10-16), in its order and types.
struct Camera {
  float rotation[9];     // scene -> camera, row-major
  float translation[3];  // scene -> camera
  float position[3];     // camera centre in scene coordinates
  float fx, fy, cx, cy;
  uint32_t width, height;
};

// Declarations of engine/include/gs/train_selftest.h:32-40 (defaults dropped).
double reference_loss(const Camera& camera, const std::vector<double>& params, const std::vector<double>& sh,
                      int sh_stride, int sh_degree, const std::vector<uint8_t>& target, const float background[3],
                      bool masked, double lambda_dssim, std::vector<double>* image, const double* head);
double reference_ssim(const std::vector<double>& x, const std::vector<double>& y, uint32_t width, uint32_t height,
                      const std::vector<double>* weights);

}  // namespace gs

// engine/src/train_selftest.cpp:27-283: opens `namespace gs`, which the line after closes.
#include "train_selftest_cpu.inc"
}  // namespace gs

namespace {

// The oracle's camera vector (oracle/gs_oracle.h gso_reference_loss): rotation[9],
// translation[3], position[3], fx, fy, cx, cy, all double; the reference stores floats.
gs::Camera make_camera(const double* c, uint32_t width, uint32_t height) {
  gs::Camera cam{};
  for (int k = 0; k < 9; ++k) cam.rotation[k] = float(c[k]);
  for (int k = 0; k < 3; ++k) cam.translation[k] = float(c[9 + k]);
  for (int k = 0; k < 3; ++k) cam.position[k] = float(c[12 + k]);
  cam.fx = float(c[15]);
  cam.fy = float(c[16]);
  cam.cx = float(c[17]);
  cam.cy = float(c[18]);
  cam.width = width;
  cam.height = height;
  return cam;
}

}  // namespace

extern "C" {

// gs::reference_loss with the oracle's argument layout. `image` (optional) receives the
// rendered FP64 image, 3 doubles per pixel.
double gsr_reference_loss(const double* camera, uint32_t width, uint32_t height, const double* params,
                          const double* sh, uint32_t n, int stride, int degree, const uint8_t* target,
                          const float* bg, int masked, double lambda, double* image, const double* head) {
  const gs::Camera cam = make_camera(camera, width, height);
  std::vector<double> p(params, params + size_t(n) * 16u);
  // The reference indexes &sh[i * stride] for every slot; keep one element when stride is 0.
  std::vector<double> s(std::max<size_t>(size_t(n) * size_t(stride), 1), 0.0);
  if (stride > 0) std::copy(sh, sh + size_t(n) * size_t(stride), s.begin());
  std::vector<uint8_t> t(target, target + size_t(width) * height * 4u);
  std::vector<double> img;
  const double loss = gs::reference_loss(cam, p, s, stride, degree, t, bg, masked != 0, lambda,
                                         image ? &img : nullptr, head);
  if (image) std::copy(img.begin(), img.end(), image);
  return loss;
}

// gs::reference_ssim (x, y: 3 doubles per pixel; weights: one per pixel or null).
double gsr_reference_ssim(const double* x, const double* y, uint32_t width, uint32_t height, const double* weights) {
  const size_t n = size_t(width) * height;
  std::vector<double> xv(x, x + n * 3u), yv(y, y + n * 3u), wv;
  if (weights) wv.assign(weights, weights + n);
  return gs::reference_ssim(xv, yv, width, height, weights ? &wv : nullptr);
}

}  // extern "C"
