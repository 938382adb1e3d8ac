// Posed training images: the reference engine's Dataset (engine/include/gs/dataset.h),
// plus synthetic orbit captures rendered on the GPU from a known scene.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "gs/camera.h"
#include "gs/splat_scene.h"

namespace gs {

struct DatasetFrame {
  std::string name;
  float c2w[16];              // camera-to-world, OpenGL convention, row-major
  std::vector<uint8_t> rgba;  // training resolution; alpha = subject mask (255 without masks)
  bool holdout = false;       // reserved for evaluation
  // A frame of its own resolution (0: the dataset's width, height and intrinsics). The
  // reference's datasets share one resolution; batched training mixes them.
  uint32_t width = 0, height = 0;
  float fx = 0, fy = 0, cx = 0, cy = 0;
  // Optional depth map (its own, usually lower, resolution): metres along the optical
  // axis, 0 where missing, with an optional confidence per sample (0..255).
  uint32_t depth_width = 0, depth_height = 0;
  std::vector<float> depth;
  std::vector<uint8_t> depth_confidence;
};

struct Dataset {
  std::string name;
  uint32_t width = 0;  // training resolution
  uint32_t height = 0;
  float fx = 0, fy = 0, cx = 0, cy = 0;  // at training resolution
  bool has_masks = false;
  bool has_depth = false;  // some frame names a depth map
  std::vector<DatasetFrame> frames;
  std::vector<float> points;          // optional sparse point cloud, xyz
  std::vector<uint8_t> point_colors;  // rgb per point
  float camera_center[3] = {0, 0, 0};
  float camera_extent = 1.0f;  // max camera distance from camera_center, x 1.1 (3DGS "scene extent")
  float world_up[3] = {0, 1, 0};
  std::vector<std::string> skipped;  // frames left out because their files could not be read

  size_t train_count() const;
  size_t holdout_count() const;
};

// Sets camera_center (mean camera position) and camera_extent from the frames
// (dataset.cpp:66-83).
void compute_camera_bounds(Dataset& dataset);

// Loads `directory`/transforms.json (nerfstudio layout: w, h, fl_x[, fl_y, cx, cy],
// frames with file_path, transform_matrix (OpenGL camera-to-world) and optional mask_path,
// depth_file_path and depth_confidence_path; optional depth_unit_scale_factor (metres per
// depth sample, default 0.001), ply_file_path point cloud and gsplat_lab.world_up), as the
// reference's load_dataset does (dataset.cpp:85-223): images resized by area so their short
// side is `target_width` (never enlarged), masks into alpha (255 without masks), every 8th
// frame held out, unreadable frames skipped and listed (throws when fewer than 2 or half
// remain), depth kept at its own resolution. Images are PNG (8/16-bit), binary PPM/PGM or
// JPEG (decoded on the GPU by nvJPEG); depth maps are 16-bit PNG or PGM.
Dataset load_dataset(const std::string& directory, uint32_t target_width);

struct InitOptions {
  uint32_t max_gaussians = 150000;
  bool subject_only = true;     // depth points only where the frame's mask covers them (with masks)
  float min_confidence = 0.3f;  // depth samples below this confidence (0..1) are left out
  float initial_opacity = 0.2f;
  uint32_t seed = 1;
};

struct InitStats {
  std::string source;  // "depth", "points" or "random"
  size_t raw_points = 0;
  float voxel_size = 0;  // cell of the merge that brought the points under budget (0: none)
};

// Initial gaussians (SH degree 0), the reference's sources in its order of preference
// (initialize_gaussians, dataset.cpp:291-523): the training frames' depth maps
// back-projected (confident samples, inside the subject mask with subject_only), else the
// dataset's sparse points, else random points in a ball of half the camera extent around
// the cameras' centre. Over budget the points are merged per occupied cell of a grid whose
// cell size is fitted to land just under max_gaussians. They are then ordered along a
// Morton curve and given identity rotations, `initial_opacity`, and isotropic scales from
// the mean distance to their 3 nearest neighbours, clamped to [1e-4, 0.02] x the points'
// robust extent (the 0.5%..99.5% box's diagonal).
SplatScene initialize_gaussians(const Dataset& dataset, const InitOptions& options, InitStats* stats = nullptr);

// Where a standing person's head is, from points on them (estimate_head,
// dataset.cpp:252-289): the top 13% of their extent along world up, a sphere of a tenth of
// that extent around the slab's median, 8.5% of the extent below the top. Not found for
// fewer than 200 points, subjects under 1 unit tall or fewer than 20 points in the slab.
struct HeadRegion {
  bool found = false;
  float center[3] = {0, 0, 0};
  float radius = 0;
  float subject_height = 0;  // extent of the points along world up
};
HeadRegion estimate_head(const Dataset& dataset, const SplatScene& subject);
HeadRegion estimate_head(const SplatScene& subject, const float up[3]);

// Pinhole camera (scene -> camera, OpenCV convention) for a frame, at the frame's own
// resolution when it has one.
Camera dataset_camera(const Dataset& dataset, const DatasetFrame& frame);

// A synthetic orbit capture: `cameras` views evenly spaced on a circle of `radius` at
// `height` around the origin, all looking at it; each view's resolution drawn from
// `resolutions` with the given probabilities (std::mt19937_64 seeded with `seed`), focal
// lengths scaled with the short side; every `holdout_every`-th view held out (0: none).
// Targets are `truth` rendered on `device` over black (alpha 255).
struct Resolution {
  uint32_t width, height;
  float focal;
  float probability;
};
struct OrbitCaptureOptions {
  uint32_t cameras = 60;
  float radius = 3.0f, height = 0.5f;
  std::vector<Resolution> resolutions = {{360, 640, 500.0f, 1.0f}};
  uint32_t holdout_every = 8;
  uint64_t seed = 7;
  int device = 0;
};
Dataset make_orbit_capture(const SplatScene& truth, const OrbitCaptureOptions& options);

}  // namespace gs
