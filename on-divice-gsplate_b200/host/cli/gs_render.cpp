// Renders a splat file headless through the training rasteriser's forward pass (the
// reference's gs_render, engine/cli/gs_render.cpp, without its graphics stack).
//
// Usage:
//   gs_render <scene.ply> <out.ppm> [width height yaw_deg pitch_deg] [--background r,g,b]
//       one orbit view: around the scene's centre (per-axis median) at 2.5x its 90th
//       percentile radius, 50 degrees across the short side; RDF scenes are turned Y-up
//   gs_render <scene.ply> --views <cameras.txt> <out_dir> [--background r,g,b]
//       one image per line of cameras.txt, written as out_dir/view_00000.ppm, ...
//       Each line: width height fx fy cx cy, then the 3x4 world-to-camera matrix
//       (OpenCV convention: x right, y down, z forward) row by row, in scene coordinates.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../src/frame.h"
#include "gs/camera.h"
#include "gs/splat_scene.h"
#include "gs_cuda.h"

namespace {

void write_ppm(const std::string& path, const std::vector<uint8_t>& rgba, uint32_t w, uint32_t h) {
  std::string head = "P6\n" + std::to_string(w) + " " + std::to_string(h) + "\n255\n";
  std::vector<uint8_t> out(head.begin(), head.end());
  out.reserve(out.size() + size_t(w) * h * 3);
  for (size_t p = 0; p < size_t(w) * h; ++p) out.insert(out.end(), &rgba[p * 4], &rgba[p * 4] + 3);
  gs::write_file(path, out);
}

std::vector<gs::Camera> read_cameras(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::vector<gs::Camera> cams;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream w(line);
    gs::Camera c{};
    float m[12];
    if (!(w >> c.width >> c.height >> c.fx >> c.fy >> c.cx >> c.cy)) throw std::runtime_error("bad camera line");
    for (float& v : m)
      if (!(w >> v)) throw std::runtime_error("bad camera line: needs 18 numbers");
    for (int r = 0; r < 3; ++r) {
      for (int k = 0; k < 3; ++k) c.rotation[r * 3 + k] = m[r * 4 + k];
      c.translation[r] = m[r * 4 + 3];
    }
    for (int k = 0; k < 3; ++k)  // centre = -R^T t
      c.position[k] = -(c.rotation[0 * 3 + k] * c.translation[0] + c.rotation[1 * 3 + k] * c.translation[1] +
                        c.rotation[2 * 3 + k] * c.translation[2]);
    cams.push_back(c);
  }
  return cams;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr,
                 "usage: %s <scene.ply> <out.ppm> [w h yaw pitch] [--background r,g,b]\n"
                 "       %s <scene.ply> --views <cameras.txt> <out_dir> [--background r,g,b]\n",
                 argv[0], argv[0]);
    return 2;
  }
  gs_context* ctx = nullptr;
  try {
    const std::vector<uint8_t> bytes = gs::read_file(argv[1]);
    gs::SplatScene scene = gs::load_splat_file(bytes.data(), bytes.size());
    std::printf("loaded %u splats, sh degree %d\n", scene.count, scene.sh_degree);
    float bg[3] = {0.0f, 0.0f, 0.0f};
    std::vector<std::string> positional;
    const std::string mode = argv[2];
    for (int i = 3; i < argc; ++i) {
      const std::string a = argv[i];
      if (a == "--background" && i + 1 < argc) {
        if (std::sscanf(argv[++i], "%f,%f,%f", &bg[0], &bg[1], &bg[2]) != 3)
          throw std::runtime_error("--background needs r,g,b");
      } else {
        positional.push_back(a);
      }
    }
    std::vector<gs::Camera> cams;
    std::vector<std::string> outputs;
    if (mode == "--views") {
      if (positional.size() < 2) throw std::runtime_error("--views needs <cameras.txt> <out_dir>");
      cams = read_cameras(positional[0]);
      for (size_t i = 0; i < cams.size(); ++i) {
        char name[32];
        std::snprintf(name, sizeof(name), "/view_%05zu.ppm", i);
        outputs.push_back(positional[1] + name);
      }
    } else {
      gs::convert_convention(scene, gs::AxisConvention::RUB);
      const uint32_t w = positional.size() > 0 ? uint32_t(std::atoi(positional[0].c_str())) : 800;
      const uint32_t h = positional.size() > 1 ? uint32_t(std::atoi(positional[1].c_str())) : 600;
      const float yaw = positional.size() > 2 ? float(std::atof(positional[2].c_str())) * 3.14159265f / 180.0f : 0.0f;
      const float pitch = positional.size() > 3 ? float(std::atof(positional[3].c_str())) * 3.14159265f / 180.0f : 0.25f;
      const gs::SceneBounds b = gs::compute_bounds(scene);
      const float d = 2.5f * b.radius;
      const float eye[3] = {b.center[0] + d * std::cos(pitch) * std::sin(yaw), b.center[1] + d * std::sin(pitch),
                            b.center[2] + d * std::cos(pitch) * std::cos(yaw)};
      float c2w[16];
      gs::look_at_c2w_gl(eye, b.center, c2w);
      const float f = 0.5f * float(std::min(w, h)) / std::tan(25.0f * 3.14159265f / 180.0f);
      cams.push_back(gs::camera_from_c2w_gl(c2w, f, f, 0.5f * float(w), 0.5f * float(h), w, h));
      outputs.push_back(mode);
    }
    gs::detail::check_status(gs_create(0, &ctx), "gs_create");
    const uint32_t stride = uint32_t(gs::sh_rest_coeffs(scene.sh_degree) * 3);
    std::vector<float> p, sh;
    gs::detail::pack_params(scene, scene.sh_degree, stride, p, sh);
    gs::detail::check_status(
        gs_model_init(ctx, std::max(scene.count, 1u), stride, p.data(), stride ? sh.data() : nullptr, scene.count),
        "gs_model_init");
    for (size_t i = 0; i < cams.size(); ++i) {
      gs_frame_data f;
      gs::detail::frame_geometry(f, cams[i], scene.count, stride, scene.sh_degree, 0u, bg);
      std::vector<uint8_t> rgba(size_t(cams[i].width) * cams[i].height * 4);
      gs::detail::check_status(gs_render(ctx, &f, rgba.data()), "gs_render");
      write_ppm(outputs[i], rgba, cams[i].width, cams[i].height);
    }
    std::printf("rendered %zu view(s)\n", cams.size());
  } catch (const std::exception& e) {
    if (ctx) gs_destroy(ctx);
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  gs_destroy(ctx);
  return 0;
}
