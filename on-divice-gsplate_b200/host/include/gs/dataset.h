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
};

struct Dataset {
  std::string name;
  uint32_t width = 0;  // training resolution
  uint32_t height = 0;
  float fx = 0, fy = 0, cx = 0, cy = 0;  // at training resolution
  bool has_masks = false;
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
// frames with file_path, transform_matrix (OpenGL camera-to-world) and optional
// mask_path; optional ply_file_path point cloud and gsplat_lab.world_up), as the
// reference's load_dataset does (dataset.cpp:85-223): images resized by area so their
// short side is `target_width` (never enlarged), masks into alpha (255 without masks),
// every 8th frame held out, unreadable frames skipped and listed (throws when fewer than
// 2 or half remain). Images are PNG (8/16-bit) or binary PPM/PGM; JPEG frames and depth
// maps are not decoded by libgs_host (JPEG frames are skipped like unreadable ones).
Dataset load_dataset(const std::string& directory, uint32_t target_width);

struct InitOptions {
  uint32_t max_gaussians = 150000;
  float initial_opacity = 0.2f;
  uint32_t seed = 1;
};

struct InitStats {
  std::string source;  // "points" or "random"
  size_t raw_points = 0;
  float voxel_size = 0;
};

// Initial gaussians (SH degree 0) from the dataset's sparse points, or random points
// around the cameras' centre (initialize_gaussians, dataset.cpp:291-523 without its depth
// source): over budget the points are merged per voxel (cell size bisected in log space to
// land under max_gaussians; the bracket widens until it does), ordered along a Morton curve, given isotropic scales from the
// mean distance to their 3 nearest neighbours (clamped to [1e-4, 0.02] x the points'
// robust extent), identity rotations and `initial_opacity`.
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
