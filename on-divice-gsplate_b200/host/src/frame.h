// Internal: FrameData and parameter packing for libgs_cuda.
#pragma once

#include <cstdint>
#include <vector>

#include "gs/camera.h"
#include "gs/splat_scene.h"
#include "gs/trainer.h"
#include "gs_cuda.h"

namespace gs::detail {

// The camera, image, model and background words of FrameData (Trainer::write_frame,
// trainer.cpp:440-470); the caller fills the schedule words. `flags` are GS_FLAG_*.
void frame_geometry(gs_frame_data& f, const Camera& camera, uint32_t slots, uint32_t sh_stride, int active_degree,
                    uint32_t flags, const float background[3]);

// The schedule words of FrameData for `step` (write_frame, trainer.cpp:495-529): learning
// rates (position decaying exponentially, times the camera extent), Adam constants and
// bias corrections, densification thresholds and seed, loss weight and SSIM constants.
void frame_schedule(gs_frame_data& f, const TrainOptions& options, uint32_t step, float camera_extent, float lambda);

// The exposure and head words of FrameData (write_frame, trainer.cpp:444, 531-544): the
// photo is divided by `gain` (null: 1); a head region in front of the camera gives its
// projected centre and radius, weighted head_weight unless it fills much of the view.
void frame_refinement(gs_frame_data& f, const Camera& camera, const HeadRegion& head, float head_weight,
                      const float* gain);

// The scene in libgs_cuda's layout (the Trainer constructor's upload, trainer.cpp:388-417):
// 16 floats per slot (position + opacity logit, log scale + alive flag, quaternion, DC)
// and sh_stride floats of SH beyond DC, the scene's coefficients up to `degree`.
void pack_params(const SplatScene& scene, int degree, uint32_t sh_stride, std::vector<float>& params16,
                 std::vector<float>& sh);

// Throws std::runtime_error carrying gs_last_error() when `code` is not GS_OK.
void check_status(int code, const char* what);

}  // namespace gs::detail
