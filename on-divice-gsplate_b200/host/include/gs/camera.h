// Pinhole cameras: the reference engine's gs::Camera (engine/include/gs/camera.h).
#pragma once

#include <cstdint>

namespace gs {

// Pinhole camera in scene coordinates, OpenCV convention (x right, y down, z forward).
struct Camera {
  float rotation[9];     // scene -> camera, row-major
  float translation[3];  // scene -> camera
  float position[3];     // camera centre in scene coordinates
  float fx, fy, cx, cy;
  uint32_t width, height;
};

// OpenGL camera-to-world (row-major 4x4) looking from `eye` at `target` with world up
// +y (the construction of train_selftest.cpp:152-174).
void look_at_c2w_gl(const float eye[3], const float target[3], float c2w[16]);

// OpenGL camera-to-world -> OpenCV world-to-camera (dataset_camera, dataset.cpp:226-250).
Camera camera_from_c2w_gl(const float c2w[16], float fx, float fy, float cx, float cy, uint32_t width,
                          uint32_t height);

}  // namespace gs
