/*
 * CPU oracle for the 3D Gaussian Splatting training step — TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker for the CUDA path, never the thing measured or shipped.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference leg may
 * load it. It restates, in plain C, the reference engine's GLSL training passes
 * (engine/shaders/train_*.comp, train_common.glsl) in fp32 with no floating-point
 * contraction, and its FP64 CPU forward + loss (engine/src/train_selftest.cpp:38-283).
 *
 * Parity pinning: the reference's FP64 CPU forward + loss (train_selftest.cpp:27-283) is
 * compiled from a reference checkout into oracle/_ref/libgs_ref.so (Makefile `ref`,
 * ref_shim.cpp). tests/test_oracle_ref.py checks that gso_reference_loss and
 * gso_reference_ssim reproduce it bit for bit (loss, FP64 image, SSIM) on the reference's own
 * test scene and on workload-shaped scenes, that the fp32 passes here render within its
 * 2.5/255 image and 1e-4 loss bars (test_trainer.cpp:34-35), and that the analytic gradients
 * pass its finite-difference rule (train_selftest.cpp:418-446) against central differences
 * of the reference's own loss. The reference has no CPU code for the sort, the backward,
 * Adam or densify (its GPU path is Vulkan, which cannot run here); those passes are pinned by
 * the reference's known-answer tests, restated in tests/test_oracle.py: pair order
 * (test_trainer.cpp:197-233), footprint exactness (test_trainer.cpp:235-289), densify
 * capacity (test_trainer.cpp:866-888), the stable depth sort (test_engine.cpp:27-68) and the
 * SSIM window constants (train_common.glsl:61-62 vs train_selftest.cpp:176-181).
 *
 * Layouts are the reference's: 16 floats of parameters per slot (train_common.glsl:3-8),
 * `sh_stride` floats of SH beyond DC per slot ([coeff][rgb]), 16 floats of projected
 * splat per slot (train_common.glsl:9-13), 12 floats of gradient per pair
 * (train_common.glsl:223-227).
 */
#ifndef GS_ORACLE_H
#define GS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-step constants; the layout of FrameData (train_common.glsl:15-37). 256 bytes. */
typedef struct gso_frame {
  float rot[3][4];     /* world -> camera rotation rows (OpenCV axes), w = translation */
  float cam_pos[4];    /* camera centre (world) */
  float intrinsics[4]; /* fx, fy, cx, cy */
  uint32_t image[4];   /* width, height, tiles_x, tiles_y */
  uint32_t model[4];   /* slots in use, active SH degree, sh_stride, flags */
  float background[4]; /* rgb, loss scale 1 / (3 W H) */
  float lr0[4];        /* position, log scale, rotation, opacity */
  float lr1[4];        /* SH DC, SH rest */
  float adam[4];       /* beta1, beta2, epsilon */
  float bias[4];       /* 1 / (1 - beta1^t), 1 / (1 - beta2^t) */
  float densify0[4];   /* grad threshold, clone max scale, prune min opacity, prune max world scale */
  float densify1[4];   /* prune max screen radius, seed (uint bits), split scale divisor */
  uint32_t limits[4];  /* pair capacity, -, -, most pairs the update accepts */
  float loss[4];       /* lambda, C1, C2 */
  float head[4];       /* head centre x, y, radius (px; 0 none), weight */
  float exposure[4];   /* rgb: 1 / gain */
} gso_frame;

#define GSO_FLAG_MASKED 1u
#define GSO_FLAG_SSIM 4u
#define GSO_FLAG_SPARSE_ADAM 128u

/* train_project.comp:26-112. projected: 16 floats per slot. */
void gso_project(const gso_frame* f, const float* params, const float* sh, uint32_t n, float* projected,
                 uint32_t* tiles, uint32_t* depth_keys);

/* The tile walk of train_emit.comp:36-50 (train_common.glsl:176-213) over stored projected records: tile counts. */
void gso_footprint_counts(const gso_frame* f, const float* projected, uint32_t n, uint32_t* tiles);

/* Tiles of one gaussian in emission order (train_emit.comp:38-49); returns the count,
   writes at most `max` ids. */
uint32_t gso_footprint_tiles(const gso_frame* f, const float* proj16, uint32_t* out, uint32_t max);

/* Stable sort of slots by 16-bit depth key (trainer.cpp:672-679). */
void gso_depth_order(const uint32_t* depth_keys, uint32_t n, uint32_t* order);

/* train_gather + scan + train_emit (train_gather.comp:15-18, trainer.cpp:576-586,
   train_emit.comp:26-64). Returns the pair total (the scan's totals[0]); writes at most
   `capacity` pairs. offsets: per slot. mismatch: gaussians whose walk disagreed. */
uint64_t gso_emit(const gso_frame* f, const float* projected, const uint32_t* tiles, const uint32_t* order,
                  uint32_t n, uint64_t capacity, uint32_t* offsets, uint32_t* pair_tile, uint32_t* pair_gaussian,
                  float* pair_grads, uint32_t* mismatch);

/* Stable sort of the pairs by tile (trainer.cpp:689-706) and tile ranges
   (train_ranges.comp:14-29). render_order[k]: pre-sort index of the k-th pair.
   ranges: 2 per tile for num_tiles + 1 tiles (the last is the padding tile). */
void gso_sort_pairs(const uint32_t* pair_tile, uint64_t pairs, uint32_t num_tiles, uint32_t* render_order,
                    uint32_t* sorted_tile, uint32_t* ranges);

/* train_forward.comp:59-183. target: RGBA8 per pixel. pixel_grad: 4 per pixel,
   tile_loss: 16 per tile, ssim_input: 8 per pixel (render rgb, w, target rgb, 0). */
void gso_forward(const gso_frame* f, const float* projected, const uint32_t* ranges, const uint32_t* render_order,
                 const uint32_t* pair_gaussian, const uint32_t* target, float* pixel_grad, uint32_t* pixel_count,
                 uint32_t* image, float* tile_loss, uint32_t* tile_count, float* ssim_input, float* pixel_dot);

/* train_ssim.comp:49-142. ssim_maps: 9 per pixel (A rgb, B rgb, C rgb). */
void gso_ssim(const gso_frame* f, const float* ssim_input, const uint32_t* ranges, float* ssim_maps,
              float* tile_loss);

/* train_ssim_grad.comp:23-70. */
void gso_ssim_grad(const gso_frame* f, const float* ssim_input, const float* ssim_maps, const uint32_t* ranges,
                   float* pixel_grad, float* pixel_dot);

/* train_backward_serial.glsl:40-103 with GS_TILE_CUTOFF (train_backward_cut.comp):
   per pair, back to front, splat_pixel_grad (train_common.glsl:228-253) summed over the
   tile's pixels; written at the pair's pre-sort index. */
void gso_backward(const gso_frame* f, const float* projected, const uint32_t* ranges, const uint32_t* render_order,
                  const uint32_t* pair_gaussian, const float* pixel_grad, const uint32_t* pixel_count,
                  const uint32_t* tile_count, float* pair_grads);

/* train_pair_sum.comp:17-32. grad_sum: 12 per slot. */
void gso_pair_sum(uint32_t n, const uint32_t* tiles, const uint32_t* offsets, const float* pair_grads,
                  float* grad_sum);

/* train_step.glsl:72-220 without the update: the gradient of the 16 parameters and the
   colour gradient / view direction per slot (sh_input, 8 floats), plus the densification
   statistics (stats: 4 per slot, updated). grad16: 16 per slot, accumulated (+=). drew:
   bit 0 set where any pair gradient was non-zero, bit 1 where the colour gradient was. */
void gso_project_backward(const gso_frame* f, const float* params, const float* sh, const uint32_t* tiles,
                          const float* grad_sum, const float* projected, float* stats, float* grad16,
                          float* sh_input, uint8_t* drew);

/* train_step_sh.comp:32-34: the SH-rest gradient from sh_input, accumulated (+=). */
void gso_sh_gradient(const gso_frame* f, const float* params, const float* sh_input, float* grad_sh);

/* Adam of train_step.glsl:62-68, 222-236 and train_step_sh.comp:25-43 for every slot,
   from accumulated gradients. Sparse Adam skips the 16 parameters of slots without
   drew bit 0 and the SH of slots without drew bit 1. */
void gso_adam(const gso_frame* f, float* params, float* sh, float* m, float* v, float* m_sh, float* v_sh,
              const float* grad16, const float* grad_sh, const uint8_t* drew);

/* train_densify_mark.comp:22-57 with the free list compacted in slot order.
   Returns the number of free slots; counters: [0] free, [2] pruned. */
void gso_densify_mark(const gso_frame* f, float* params, float* sh, float* m, float* v, float* m_sh, float* v_sh,
                      const float* stats, uint32_t* spawn, uint32_t* free_list, uint32_t* counters);

/* train_densify_spawn.comp:38-70, spawners taken in slot order (deterministic). */
void gso_densify_spawn(const gso_frame* f, float* params, float* sh, float* m, float* v, float* m_sh, float* v_sh,
                       const uint32_t* spawn, const uint32_t* free_list, uint32_t* counters, uint32_t capacity);

/* train_reset_opacity.comp:17-23. */
void gso_reset_opacity(const gso_frame* f, float* params, float* m, float* v, float max_logit);

/* FP64 forward + loss of train_selftest.cpp:79-283 (project, stable depth sort, blend over
   all gaussians per pixel, L1 + lambda (1 - SSIM)). params: 16 doubles per slot, sh:
   `stride` doubles per slot. camera: rotation[9] row-major, translation[3], position[3],
   fx, fy, cx, cy. image: optional 3 doubles per pixel. signature: optional hash of every
   blend decision (which splats each pixel took, where it stopped, which alphas clamped,
   the depth order): central differences whose stencil changes it cross a cut-off. */
double gso_reference_loss(const double* camera, uint32_t width, uint32_t height, const double* params,
                          const double* sh, uint32_t n, int stride, int degree, const uint8_t* target,
                          const float* bg, int masked, double lambda, double* image, const double* head,
                          uint64_t* signature);

/* reference_ssim of train_selftest.cpp:176-217 (x, y: 3 doubles per pixel). */
double gso_reference_ssim(const double* x, const double* y, uint32_t width, uint32_t height, const double* weights);

/* The SSIM window the shaders hard-code (train_common.glsl:61-62). */
void gso_ssim_window(float out[11]);

/* PCG hash of train_common.glsl:145-149. */
uint32_t gso_pcg_hash(uint32_t v);

/* Threads the parallel loops use (0: all host threads). */
void gso_set_threads(int threads);
int gso_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
