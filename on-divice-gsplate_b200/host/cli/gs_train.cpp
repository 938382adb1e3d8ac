// Trains gaussians on the B200 path and writes a 3DGS .ply (the reference's gs_train,
// engine/cli/gs_train.cpp, over libgs_cuda).
//
// Usage:
//   gs_train <dataset> <out.ply> [--iters 3000] [--views-per-step 1] [--max-gaussians N] [--sh 3]
//            [--eval-every 1000] [--dssim 0.2] [--dssim-end L] [--grad-threshold 2e-4] [--opacity-reset N]
//            [--sparse-adam] [--atomic] [--no-autotune] [--seed 1] [--json <metrics.json>]
//            [--gt-gaussians N] [--init-gaussians N] [--cameras N] [--width 360] [--no-masks]
//            [--head-weight W] [--refine-poses] [--pose-lr shift,turn] [--pose-lr-final F] [--pose-from N]
//            [--eval-pose-steps N] [--pose-out poses.json] [--refine-exposure]
//            [--refine-motion] [--motion-nodes 64] [--motion-lr shift,turn] [--motion-lr-final F] [--motion-from N]
//            [--motion-reg decay,rigidity,smoothness,center] [--motion-out motion.json]
//            [--eval-rest <capture_dir>] (held-out views of a twin capture with the subject standing still:
//            the model at rest against it)
// <dataset> is a capture folder (transforms.json; PNG/PPM/JPEG images, resized so the short
// side is --width, optional depth maps; initial gaussians from the depth maps, its point
// cloud or random, up to --init-gaussians, 150000 by default; the reference's default
// options with the schedule scaled to --iters)
// or a synthetic orbit capture:
//   synthetic:orbit        ground truth of 100k gaussians (radius-1 ball, log-scales N(-4, 0.5),
//                          SH 3 ~ N(0, 0.2)), 60 cameras on a circle of radius 3 at height 0.5,
//                          360x640 f=500, every 8th held out; 20k initial gaussians at ground-truth
//                          means + N(0, 0.02) with their DC colour and fresh log-scales, rotations
//                          and opacities; learning rates of the orbit workload
//   synthetic:orbit-mixed  1M ground truth (radius-2 ball, log-scales N(-5, 0.5)), 300k initial,
//                          3M slots, 200 cameras at 360x640 / 720x1280 / 1080x1920 (0.4 / 0.4 / 0.2),
//                          focal length scaled with the short side
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "gs/dataset.h"
#include "gs/splat_scene.h"
#include "gs/trainer.h"

namespace {

struct Synthetic {
  gs::RandomSceneOptions truth;
  uint32_t init = 0;
  gs::OrbitCaptureOptions capture;
  uint32_t max_gaussians = 0;
};

Synthetic preset(const std::string& name) {
  Synthetic s;
  if (name == "orbit") {
    s.truth = {100000, 1, 3, 1.0f, -4.0f, 0.5f, 0.2f};
    s.init = 20000;
    s.capture.cameras = 60;
    s.capture.resolutions = {{360, 640, 500.0f, 1.0f}};
    s.max_gaussians = 300000;
  } else if (name == "orbit-mixed") {
    s.truth = {1000000, 1, 3, 2.0f, -5.0f, 0.5f, 0.2f};
    s.init = 300000;
    s.capture.cameras = 200;
    s.capture.resolutions = {{360, 640, 500.0f, 0.4f}, {720, 1280, 1000.0f, 0.4f}, {1080, 1920, 1500.0f, 0.2f}};
    s.max_gaussians = 3000000;
  } else {
    throw std::runtime_error("unknown synthetic dataset " + name + " (orbit, orbit-mixed)");
  }
  return s;
}

// Initial gaussians: ground-truth means + N(0, 0.02), the ground truth's DC colour, SH
// rest zero; log-scales, rotations and opacities drawn afresh from the same distributions.
gs::SplatScene initial_scene(const gs::SplatScene& truth, const gs::RandomSceneOptions& dist, uint32_t count,
                             uint64_t seed) {
  gs::RandomSceneOptions fresh = dist;
  fresh.count = count;
  fresh.seed = seed + 17;
  fresh.sh_degree = 0;
  gs::SplatScene init = gs::make_random_scene(fresh);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> noise(0.0f, 0.02f);
  std::uniform_int_distribution<uint32_t> pick(0, truth.count - 1);
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t j = count >= truth.count ? i % truth.count : pick(rng);
    for (int k = 0; k < 3; ++k) {
      init.positions[size_t(i) * 3 + k] = truth.positions[size_t(j) * 3 + k] + noise(rng);
      init.sh_dc[size_t(i) * 3 + k] = truth.sh_dc[size_t(j) * 3 + k];
    }
  }
  return init;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr,
                 "usage: %s <synthetic:orbit|synthetic:orbit-mixed> <out.ply> [--iters N] [--views-per-step K]\n"
                 "       [--max-gaussians N] [--sh D] [--eval-every N] [--dssim L] [--dssim-end L]\n"
                 "       [--grad-threshold T] [--opacity-reset N] [--sparse-adam] [--atomic] [--no-autotune]\n"
                 "       [--seed S] [--json metrics.json] [--gt-gaussians N] [--init-gaussians N] [--cameras N]\n",
                 argv[0]);
    return 2;
  }
  try {
    const std::string source = argv[1], out_path = argv[2];
    const bool synthetic = source.rfind("synthetic:", 0) == 0;
    Synthetic syn;
    gs::TrainOptions options;
    uint32_t width = 360, init_max = 150000;
    if (synthetic) {
      syn = preset(source.substr(10));
      options.lr_opacity = 5e-2f;  // the orbit workload's rates: means 1.6e-4, scales 5e-3, rot 1e-3,
      options.lr_sh_rest = 2.5e-3f;  // opacity 5e-2, SH 2.5e-3
      options.masked = false;
      options.random_background = false;
      options.lambda_dssim_end = -1.0f;
      options.densify_from = 500;
      options.densify_until = 2500;
      options.densify_interval = 100;
      options.max_gaussians = syn.max_gaussians;
    }
    uint32_t iterations = 3000, eval_every = 1000;
    std::string json_path, pose_out, motion_out, eval_rest;
    for (int i = 3; i < argc; ++i) {
      const std::string arg = argv[i];
      auto next = [&]() -> const char* {
        if (i + 1 >= argc) throw std::runtime_error(arg + " needs a value");
        return argv[++i];
      };
      if (arg == "--iters") iterations = uint32_t(std::atoi(next()));
      else if (arg == "--views-per-step") options.views_per_step = uint32_t(std::atoi(next()));
      else if (arg == "--max-gaussians") options.max_gaussians = uint32_t(std::atoi(next()));
      else if (arg == "--sh") options.sh_degree = std::atoi(next());
      else if (arg == "--eval-every") eval_every = uint32_t(std::atoi(next()));
      else if (arg == "--dssim") options.lambda_dssim = float(std::atof(next()));
      else if (arg == "--dssim-end") options.lambda_dssim_end = float(std::atof(next()));
      else if (arg == "--grad-threshold") options.densify_grad_threshold = float(std::atof(next()));
      else if (arg == "--opacity-reset") options.opacity_reset_interval = uint32_t(std::atoi(next()));
      else if (arg == "--sparse-adam") options.sparse_adam = true;
      else if (arg == "--atomic") options.deterministic = false;
      else if (arg == "--no-autotune") options.autotune = false;
      else if (arg == "--seed") options.seed = uint32_t(std::atoi(next()));
      else if (arg == "--json") json_path = next();
      else if (arg == "--gt-gaussians") syn.truth.count = uint32_t(std::atoi(next()));
      else if (arg == "--init-gaussians") syn.init = init_max = uint32_t(std::atoi(next()));
      else if (arg == "--cameras") syn.capture.cameras = uint32_t(std::atoi(next()));
      else if (arg == "--width") width = uint32_t(std::atoi(next()));
      else if (arg == "--no-masks") options.masked = false;
      else if (arg == "--head-weight") options.head_weight = float(std::atof(next()));
      else if (arg == "--refine-poses") options.refine_poses = true;
      else if (arg == "--pose-lr") {
        if (std::sscanf(next(), "%f,%f", &options.lr_pose_shift, &options.lr_pose_turn) != 2)
          throw std::runtime_error("--pose-lr needs shift,turn");
      } else if (arg == "--pose-lr-final") options.lr_pose_final = float(std::atof(next()));
      else if (arg == "--pose-from") options.pose_from = uint32_t(std::atoi(next()));
      else if (arg == "--eval-pose-steps") options.eval_pose_steps = uint32_t(std::atoi(next()));
      else if (arg == "--pose-out") pose_out = next();
      else if (arg == "--refine-exposure") options.refine_exposure = true;
      else if (arg == "--refine-motion") options.refine_motion = true;
      else if (arg == "--motion-nodes") options.motion_nodes = uint32_t(std::atoi(next()));
      else if (arg == "--motion-lr") {
        if (std::sscanf(next(), "%f,%f", &options.lr_motion_shift, &options.lr_motion_turn) != 2)
          throw std::runtime_error("--motion-lr needs shift,turn");
      } else if (arg == "--motion-lr-final") options.lr_motion_final = float(std::atof(next()));
      else if (arg == "--motion-from") options.motion_from = uint32_t(std::atoi(next()));
      else if (arg == "--motion-reg") {
        if (std::sscanf(next(), "%f,%f,%f,%f", &options.motion_decay, &options.motion_rigidity,
                        &options.motion_smoothness, &options.motion_center) != 4)
          throw std::runtime_error("--motion-reg needs decay,rigidity,smoothness,center");
      } else if (arg == "--motion-out") motion_out = next();
      else if (arg == "--eval-rest") eval_rest = next();
      else throw std::runtime_error("unknown option " + arg);
    }
    // The schedule (densify window, SH degree interval) scales with the iterations, as
    // scaled_options does for the defaults.
    const double scale = double(iterations) / 3000.0;
    options.iterations = iterations;
    options.densify_from = uint32_t(options.densify_from * scale);
    options.densify_until = uint32_t(options.densify_until * scale);
    if (synthetic) options.densify_interval = std::max(1u, uint32_t(options.densify_interval * scale));
    options.opacity_reset_interval = uint32_t(options.opacity_reset_interval * scale);
    options.sh_degree_interval = std::max(1u, uint32_t(options.sh_degree_interval * scale));
    options.retune_first = std::min(options.retune_first, iterations / 2);

    const auto t0 = std::chrono::steady_clock::now();
    gs::Dataset dataset;
    gs::SplatScene init;
    if (synthetic) {
      const gs::SplatScene truth = gs::make_random_scene(syn.truth);
      dataset = gs::make_orbit_capture(truth, syn.capture);
      init = initial_scene(truth, syn.truth, syn.init, options.seed);
    } else {
      dataset = gs::load_dataset(source, width);
      for (const std::string& s : dataset.skipped) std::printf("skipped %s\n", s.c_str());
      gs::InitOptions io;
      io.max_gaussians = init_max;
      io.seed = options.seed;
      gs::InitStats st;
      init = gs::initialize_gaussians(dataset, io, &st);
      std::printf("initial gaussians from %s: %zu points -> %u\n", st.source.c_str(), st.raw_points, init.count);
      // The head region from the subject's points (masked captures with a point cloud).
      if (options.masked && dataset.has_masks && st.source != "random") options.head = gs::estimate_head(dataset, init);
      if (options.head.found)
        std::printf("head region: centre %.2f %.2f %.2f, radius %.2f (subject %.2f tall), weight %.1f\n",
                    options.head.center[0], options.head.center[1], options.head.center[2], options.head.radius,
                    options.head.subject_height, options.head_weight);
    }
    std::printf("dataset %s: %zu views (%zu held out), camera extent %.3f; %u initial gaussians (%.1f s)\n",
                source.c_str(), dataset.frames.size(), dataset.holdout_count(), dataset.camera_extent, init.count,
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());

    gs::Dataset rest;
    if (!eval_rest.empty()) rest = gs::load_dataset(eval_rest, width);
    gs::CudaContext ctx;
    gs::Trainer trainer(ctx, std::move(dataset), init, options);
    if (options.refine_motion)
      std::printf("motion: %zu nodes from step %u\n", trainer.motion_nodes().size(), options.motion_from);
    struct Eval {
      uint32_t step;
      double psnr, train_seconds;  // training time up to this evaluation (evaluations excluded)
    };
    std::vector<Eval> evals;
    double train_s = 0.0;
    while (!trainer.finished()) {
      const uint32_t chunk = std::min(eval_every > 0 ? eval_every : iterations, iterations - trainer.stats().step);
      const auto s0 = std::chrono::steady_clock::now();
      for (uint32_t k = 0; k < chunk && !trainer.finished(); ++k) trainer.step();
      train_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
      const gs::TrainStats& s = trainer.stats();
      std::printf("step %5u  l1 %.4f  psnr %5.2f  gaussians %7u (+%u -%u)  pairs %9llu  sh %d  %.2f ms/step\n", s.step,
                  s.l1, s.psnr, s.gaussians, s.spawned, s.pruned, (unsigned long long)s.pairs, s.sh_degree, s.step_ms);
      if (options.refine_poses)
        std::printf("  poses: shift %.4f (max %.4f), turn %.3f deg (max %.3f) over %u updates\n", s.pose_shift_mean,
                    s.pose_shift_max, s.pose_turn_mean, s.pose_turn_max, s.pose_updates);
      if (options.refine_exposure)
        std::printf("  exposure: luminance gain %.3f..%.3f, tint spread %.4f over %u updates\n", s.exposure_low,
                    s.exposure_high, s.exposure_tint, s.exposure_updates);
      if (options.refine_motion)
        std::printf("  motion: shift %.4f (max %.4f), turn %.3f deg (max %.3f) over %u view updates\n",
                    s.motion_shift_mean, s.motion_shift_max, s.motion_turn_mean, s.motion_turn_max, s.motion_updates);
      const gs::EvalResult e = trainer.evaluate();
      std::printf("  eval: held-out PSNR %.2f dB, SSIM %.4f over %u views", e.psnr, e.ssim, e.views);
      if (e.aligned) std::printf(" (%.2f dB at the poses as given)", e.psnr_unaligned);
      if (e.head_views) std::printf("; head %.2f dB over %u views", e.head_psnr, e.head_views);
      std::printf("\n");
      if (!rest.frames.empty()) {
        const gs::EvalResult r = trainer.evaluate_at_rest(rest);
        std::printf("  at rest: held-out PSNR %.2f dB, SSIM %.4f over %u views\n", r.psnr, r.ssim, r.views);
      }
      evals.push_back({s.step, e.psnr, train_s});
    }
    const gs::TrainStats& s = trainer.stats();
    const double views_per_s = double(s.views) / train_s;
    std::printf("trained %u steps, %llu views in %.1f s: %.1f views/s; tuning %s\n", s.step,
                (unsigned long long)s.views, train_s, views_per_s, trainer.reduction().c_str());
    if (!pose_out.empty()) {
      // Every frame's camera-to-world (OpenGL axes, row-major) after refinement.
      std::ofstream poses(pose_out);
      poses.precision(9);
      poses << "{\"frames\": [";
      const gs::Dataset& d = trainer.dataset();
      for (size_t f = 0; f < d.frames.size(); ++f) {
        const gs::Camera c = trainer.camera_for(f);
        poses << (f ? "," : "") << "\n{\"file_path\": \"" << d.frames[f].name
              << "\", \"holdout\": " << (d.frames[f].holdout ? "true" : "false") << ", \"transform_matrix\": [";
        // Columns R^T e0, -R^T e1, -R^T e2 (OpenCV to OpenGL axes) and the centre.
        for (int r = 0; r < 3; ++r)
          poses << (r ? "," : "") << "[" << c.rotation[r] << "," << -c.rotation[3 + r] << ","
                << -c.rotation[6 + r] << "," << c.position[r] << "]";
        poses << ",[0,0,0,1]]}";
      }
      poses << "\n]}\n";
    }
    if (!motion_out.empty()) {
      // The nodes at rest (x, y, z, radius) and every view's motion of each: turn (axis-angle) and shift.
      std::ofstream m(motion_out);
      m.precision(7);
      m << "{\"nodes\": [";
      const auto& nodes = trainer.motion_nodes();
      for (size_t k = 0; k < nodes.size(); ++k)
        m << (k ? "," : "") << "[" << nodes[k].position[0] << "," << nodes[k].position[1] << ","
          << nodes[k].position[2] << "," << nodes[k].radius << "]";
      m << "],\n\"frames\": [";
      for (size_t f = 0; f < trainer.dataset().frames.size(); ++f) {
        std::string turns, shifts;
        for (size_t k = 0; k < nodes.size(); ++k) {
          float turn[3], shift[3];
          trainer.node_motion(f, uint32_t(k), turn, shift);
          char buf[128];
          std::snprintf(buf, sizeof(buf), "%s[%.7g,%.7g,%.7g]", k ? "," : "", turn[0], turn[1], turn[2]);
          turns += buf;
          std::snprintf(buf, sizeof(buf), "%s[%.7g,%.7g,%.7g]", k ? "," : "", shift[0], shift[1], shift[2]);
          shifts += buf;
        }
        m << (f ? "," : "") << "\n{\"holdout\": " << (trainer.dataset().frames[f].holdout ? "true" : "false")
          << ", \"turn\": [" << turns << "], \"shift\": [" << shifts << "]}";
      }
      m << "\n]}\n";
    }
    gs::SplatScene out = trainer.export_scene();
    gs::convert_convention(out, gs::AxisConvention::RDF);  // what .ply readers expect
    gs::write_file(out_path, gs::save_ply(out));
    std::printf("wrote %s: %u gaussians\n", out_path.c_str(), out.count);
    if (!json_path.empty()) {
      std::ofstream j(json_path);
      j << "{\"dataset\": \"" << source << "\", \"iterations\": " << s.step
        << ", \"views_per_step\": " << options.views_per_step << ", \"views\": " << s.views
        << ", \"train_seconds\": " << train_s << ", \"views_per_s\": " << views_per_s
        << ", \"final_psnr\": " << (evals.empty() ? 0.0 : evals.back().psnr) << ", \"gaussians\": " << s.gaussians
        << ", \"spawned\": " << s.spawned << ", \"pruned\": " << s.pruned
        << ", \"overflow_steps\": " << s.overflow_steps << ", \"tuning\": \"" << trainer.reduction()
        << "\", \"eval\": [";
      for (size_t k = 0; k < evals.size(); ++k)
        j << (k ? ", " : "") << "{\"step\": " << evals[k].step << ", \"psnr\": " << evals[k].psnr
          << ", \"train_seconds\": " << evals[k].train_seconds << "}";
      j << "]}\n";
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
