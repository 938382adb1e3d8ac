/*
 * CPU oracle for the 3DGS training step — TEST INFRASTRUCTURE ONLY (see gs_oracle.h).
 * Built with -ffp-contract=off so every float operation rounds as written, mirroring the
 * `precise` arithmetic of the reference's footprint helpers. Each function cites the
 * reference file:line it restates. Parallel loops write disjoint outputs, so results do
 * not depend on the thread count.
 */
#include "gs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TILE 16u
static const float kNear = 0.02f;
static const float kLogRange = 15.6096404744f; /* log2(kFar / kNear), kFar = 1000 (train_common.glsl:65-66) */
static const float kDilation = 0.3f;
static const float kMinAlpha = 1.0f / 255.0f;
static const float kMaxAlpha = 0.99f;
static const float kMinTransmittance = 1e-4f;

/* train_common.glsl:61-62 */
static const float kSsimWindow[11] = {0.001028380f, 0.007598758f, 0.036000772f, 0.109360690f,
                                      0.213005538f, 0.266011725f, 0.213005538f, 0.109360690f,
                                      0.036000772f, 0.007598758f, 0.001028380f};

static int g_threads = 0;
void gso_set_threads(int threads) { g_threads = threads; }
int gso_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}
#define PAR_FOR _Pragma("omp parallel for schedule(dynamic, 64) num_threads(gso_get_threads())")

void gso_ssim_window(float out[11]) { memcpy(out, kSsimWindow, sizeof(kSsimWindow)); }

static float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
static int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
static float sigmoidf(float x) { return 1.0f / (1.0f + expf(-x)); }

/* train_common.glsl:72-78; R[row][col]. */
static void quat_to_matrix(const float q[4], float R[3][3]) {
  const float w = q[0], x = q[1], y = q[2], z = q[3];
  R[0][0] = 1.0f - 2.0f * (y * y + z * z);
  R[1][0] = 2.0f * (x * y + w * z);
  R[2][0] = 2.0f * (x * z - w * y);
  R[0][1] = 2.0f * (x * y - w * z);
  R[1][1] = 1.0f - 2.0f * (x * x + z * z);
  R[2][1] = 2.0f * (y * z + w * x);
  R[0][2] = 2.0f * (x * z + w * y);
  R[1][2] = 2.0f * (y * z - w * x);
  R[2][2] = 1.0f - 2.0f * (x * x + y * y);
}

static int sh_rest_coeffs(uint32_t degree) { return degree == 0u ? 0 : (int)((degree + 1u) * (degree + 1u)) - 1; }

/* train_common.glsl:84-109 */
static void sh_basis(const float d[3], uint32_t degree, float b[16]) {
  const float x = d[0], y = d[1], z = d[2];
  for (int k = 0; k < 16; ++k) b[k] = 0.0f;
  b[0] = 0.28209479177387814f;
  if (degree >= 1u) {
    b[1] = -0.4886025119029199f * y;
    b[2] = 0.4886025119029199f * z;
    b[3] = -0.4886025119029199f * x;
  }
  if (degree >= 2u) {
    const float xx = x * x, yy = y * y, zz = z * z;
    b[4] = 1.0925484305920792f * x * y;
    b[5] = -1.0925484305920792f * y * z;
    b[6] = 0.31539156525252005f * (2.0f * zz - xx - yy);
    b[7] = -1.0925484305920792f * x * z;
    b[8] = 0.5462742152960396f * (xx - yy);
    if (degree >= 3u) {
      b[9] = -0.5900435899266435f * y * (3.0f * xx - yy);
      b[10] = 2.890611442640554f * x * y * z;
      b[11] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
      b[12] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
      b[13] = -0.4570457994644658f * x * (4.0f * zz - xx - yy);
      b[14] = 1.445305721320277f * z * (xx - yy);
      b[15] = -0.5900435899266435f * x * (xx - 3.0f * yy);
    }
  }
}

/* train_common.glsl:111-140; g[k][axis]. */
static void sh_basis_grad(const float d[3], uint32_t degree, float g[16][3]) {
  const float x = d[0], y = d[1], z = d[2];
  memset(g, 0, sizeof(float) * 48);
  if (degree >= 1u) {
    const float C1 = 0.4886025119029199f;
    g[1][1] = -C1;
    g[2][2] = C1;
    g[3][0] = -C1;
  }
  if (degree >= 2u) {
    const float xx = x * x, yy = y * y, zz = z * z;
    const float A = 1.0925484305920792f, B = 0.31539156525252005f, C = 0.5462742152960396f;
    g[4][0] = A * y; g[4][1] = A * x; g[4][2] = 0.0f;
    g[5][0] = 0.0f; g[5][1] = -A * z; g[5][2] = -A * y;
    g[6][0] = B * (-2.0f * x); g[6][1] = B * (-2.0f * y); g[6][2] = B * (4.0f * z);
    g[7][0] = -A * z; g[7][1] = 0.0f; g[7][2] = -A * x;
    g[8][0] = C * (2.0f * x); g[8][1] = C * (-2.0f * y); g[8][2] = 0.0f;
    if (degree >= 3u) {
      const float D = -0.5900435899266435f, E = 2.890611442640554f, F = -0.4570457994644658f;
      const float G = 0.3731763325901154f, H = 1.445305721320277f;
      g[9][0] = D * (6.0f * x * y); g[9][1] = D * (3.0f * xx - 3.0f * yy); g[9][2] = 0.0f;
      g[10][0] = E * (y * z); g[10][1] = E * (x * z); g[10][2] = E * (x * y);
      g[11][0] = F * (-2.0f * x * y); g[11][1] = F * (4.0f * zz - xx - 3.0f * yy); g[11][2] = F * (8.0f * y * z);
      g[12][0] = G * (-6.0f * x * z); g[12][1] = G * (-6.0f * y * z); g[12][2] = G * (6.0f * zz - 3.0f * xx - 3.0f * yy);
      g[13][0] = F * (4.0f * zz - 3.0f * xx - yy); g[13][1] = F * (-2.0f * x * y); g[13][2] = F * (8.0f * x * z);
      g[14][0] = H * (2.0f * x * z); g[14][1] = H * (-2.0f * y * z); g[14][2] = H * (xx - yy);
      g[15][0] = D * (3.0f * xx - 3.0f * yy); g[15][1] = D * (-6.0f * x * y); g[15][2] = 0.0f;
    }
  }
}

/* train_common.glsl:145-149 */
uint32_t gso_pcg_hash(uint32_t v) {
  const uint32_t state = v * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

/* train_common.glsl:151-161 */
static float uniform01(uint32_t* state) {
  *state = gso_pcg_hash(*state);
  return (float)(*state >> 8u) * (1.0f / 16777216.0f);
}
static void normal3(uint32_t* state, float out[3]) {
  const float u1 = fmaxf(uniform01(state), 1e-7f), u2 = uniform01(state);
  const float u3 = fmaxf(uniform01(state), 1e-7f), u4 = uniform01(state);
  const float r1 = sqrtf(-2.0f * logf(u1)), r2 = sqrtf(-2.0f * logf(u3));
  out[0] = r1 * cosf(6.283185307f * u2);
  out[1] = r1 * sinf(6.283185307f * u2);
  out[2] = r2 * cosf(6.283185307f * u4);
}

/* train_common.glsl:169-172 */
static float footprint_threshold(float opacity) {
  const float t = 2.0f * logf(opacity * 255.0f);
  return t * 1.0001f + 1e-4f;
}

/* train_common.glsl:176-181 */
static void footprint_pixels(float lo, float hi, uint32_t size, int out[2]) {
  const int n = (int)size;
  out[0] = clampi((int)clampf(ceilf(lo), -1.0f, (float)n), 0, n);
  out[1] = clampi((int)clampf(floorf(hi), -1.0f, (float)n), -1, n - 1);
}

/* train_common.glsl:185-190 */
static void footprint_rows(const float m[2], const float cov[3], float t, uint32_t height, int out[2]) {
  const float ey = sqrtf(t * cov[2]);
  const float v = m[1] - 0.5f;
  const float lo = v - ey, hi = v + ey;
  footprint_pixels(lo, hi, height, out);
}

/* train_common.glsl:193-213; returns [x0, x1) in out. */
static void footprint_row_tiles(const float m[2], const float cov[3], float t, const int rows[2], uint32_t ty,
                                uint32_t width, uint32_t out[2]) {
  const float u = m[0] - 0.5f, v = m[1] - 0.5f;
  const int r0 = (int)(ty * TILE) > rows[0] ? (int)(ty * TILE) : rows[0];
  const int r1 = (int)(ty * TILE + TILE - 1u) < rows[1] ? (int)(ty * TILE + TILE - 1u) : rows[1];
  const float y0 = (float)r0 - v;
  const float y1 = (float)r1 - v;
  const float a = cov[0], b = cov[1], c = cov[2];
  const float k = b / c;
  const float w = (a * c - b * b) / c;
  const float side = b * sqrtf(t / a);
  const float dr = clampf(side, y0, y1);
  const float dl = clampf(-side, y0, y1);
  const float x_max = k * dr + sqrtf(fmaxf(w * (t - dr * dr / c), 0.0f));
  const float x_min = k * dl - sqrtf(fmaxf(w * (t - dl * dl / c), 0.0f));
  const float lo = u + x_min, hi = u + x_max;
  int cols[2];
  footprint_pixels(lo, hi, width, cols);
  if (cols[0] > cols[1]) {
    out[0] = out[1] = 0u;
    return;
  }
  out[0] = (uint32_t)cols[0] / TILE;
  out[1] = (uint32_t)cols[1] / TILE + 1u;
}

static uint32_t walk_count(const gso_frame* f, const float m[2], const float cov[3], float thr) {
  int rows[2];
  uint32_t tiles = 0u;
  footprint_rows(m, cov, thr, f->image[1], rows);
  if (rows[0] <= rows[1]) {
    for (uint32_t ty = (uint32_t)rows[0] / TILE; ty <= (uint32_t)rows[1] / TILE; ++ty) {
      uint32_t span[2];
      footprint_row_tiles(m, cov, thr, rows, ty, f->image[0], span);
      tiles += span[1] - span[0];
    }
  }
  return tiles;
}

/* train_project.comp:26-112 (without subject motion). */
void gso_project(const gso_frame* f, const float* params, const float* sh, uint32_t n, float* projected,
                 uint32_t* tiles_out, uint32_t* depth_keys) {
  PAR_FOR
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const uint32_t i = (uint32_t)ii;
    const float* p = params + (size_t)i * 16u;
    float out[16] = {0};
    uint32_t tiles = 0u;
    float t[3];
    for (int r = 0; r < 3; ++r) t[r] = f->rot[r][0] * p[0] + f->rot[r][1] * p[1] + f->rot[r][2] * p[2] + f->rot[r][3];
    const float opacity = sigmoidf(p[3]);
    if (p[7] > 0.5f && t[2] > kNear && opacity >= kMinAlpha) {
      const float fx = f->intrinsics[0], fy = f->intrinsics[1], cx = f->intrinsics[2], cy = f->intrinsics[3];
      const float width = (float)f->image[0], height = (float)f->image[1];
      const float inv_z = 1.0f / t[2];
      const float mean[2] = {fx * t[0] * inv_z + cx, fy * t[1] * inv_z + cy};
      const float lim_x = 1.3f * fmaxf(cx, width - cx) / fx;
      const float lim_y = 1.3f * fmaxf(cy, height - cy) / fy;
      const float tx = clampf(t[0] * inv_z, -lim_x, lim_x);
      const float ty = clampf(t[1] * inv_z, -lim_y, lim_y);
      /* J rows (third row zero): (fx/z, 0, -fx tx/z), (0, fy/z, -fy ty/z) */
      const float j00 = fx * inv_z, j02 = -fx * tx * inv_z, j11 = fy * inv_z, j12 = -fy * ty * inv_z;
      float T[2][3];
      for (int c = 0; c < 3; ++c) {
        T[0][c] = j00 * f->rot[0][c] + j02 * f->rot[2][c];
        T[1][c] = j11 * f->rot[1][c] + j12 * f->rot[2][c];
      }
      const float* q = p + 8;
      const float qlen = fmaxf(sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), 1e-12f);
      const float qn[4] = {q[0] / qlen, q[1] / qlen, q[2] / qlen, q[3] / qlen};
      float R[3][3];
      quat_to_matrix(qn, R);
      const float s[3] = {expf(p[4]), expf(p[5]), expf(p[6])};
      float M[3][3], Sigma[3][3];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) M[r][c] = R[r][c] * s[c];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Sigma[r][c] = M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2];
      float cov[2][2];
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          float acc = 0.0f;
          for (int k = 0; k < 3; ++k) {
            const float row = T[a][0] * Sigma[0][k] + T[a][1] * Sigma[1][k] + T[a][2] * Sigma[2][k];
            acc += row * T[b][k];
          }
          cov[a][b] = acc;
        }
      /* GLSL cov[0][1] is column 0, row 1 */
      const float a = cov[0][0] + kDilation, b = cov[1][0], c = cov[1][1] + kDilation;
      const float det = a * c - b * b;
      if (det > 0.0f) {
        const float mid = 0.5f * (a + c);
        const float lambda = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
        const float sigma = sqrtf(lambda);
        const float cov2[3] = {a, b, c};
        const float thr = footprint_threshold(opacity);
        tiles = walk_count(f, mean, cov2, thr);
        if (tiles > 0u) {
          out[12] = a;
          out[13] = b;
          out[14] = c;
          out[15] = thr;
          const uint32_t degree = f->model[1];
          const float* shp = sh + (size_t)i * f->model[2];
          float dir[3] = {p[0] - f->cam_pos[0], p[1] - f->cam_pos[1], p[2] - f->cam_pos[2]};
          const float dlen = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
          for (int k = 0; k < 3; ++k) dir[k] = dir[k] / dlen;
          float basis[16];
          sh_basis(dir, degree, basis);
          float color[3];
          for (int ch = 0; ch < 3; ++ch) color[ch] = basis[0] * p[12 + ch];
          const int coeffs = sh_rest_coeffs(degree);
          for (int k = 0; k < coeffs; ++k)
            for (int ch = 0; ch < 3; ++ch) color[ch] += basis[k + 1] * shp[k * 3 + ch];
          uint32_t clamped = 0u;
          for (int ch = 0; ch < 3; ++ch) {
            color[ch] += 0.5f;
            if (color[ch] < 0.0f) clamped |= 1u << ch;
            color[ch] = fmaxf(color[ch], 0.0f);
          }
          const float inv_det = 1.0f / det;
          out[0] = mean[0];
          out[1] = mean[1];
          out[2] = t[2];
          out[3] = opacity;
          out[4] = c * inv_det;
          out[5] = -b * inv_det;
          out[6] = a * inv_det;
          out[7] = ceilf(3.0f * sigma);
          out[8] = color[0];
          out[9] = color[1];
          out[10] = color[2];
          memcpy(&out[11], &clamped, 4);
        }
      }
    }
    memcpy(projected + (size_t)i * 16u, out, sizeof(out));
    tiles_out[i] = tiles;
    depth_keys[i] =
        tiles > 0u ? (uint32_t)(clampf(log2f(out[2] / kNear) / kLogRange, 0.0f, 1.0f) * 65535.0f) : 0xffffu;
  }
}

void gso_footprint_counts(const gso_frame* f, const float* projected, uint32_t n, uint32_t* tiles) {
  PAR_FOR
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const float* q = projected + (size_t)ii * 16u;
    tiles[ii] = q[15] == 0.0f && q[12] == 0.0f ? 0u : walk_count(f, q, q + 12, q[15]);
  }
}

uint32_t gso_footprint_tiles(const gso_frame* f, const float* q, uint32_t* out, uint32_t max) {
  int rows[2];
  uint32_t count = 0u;
  footprint_rows(q, q + 12, q[15], f->image[1], rows);
  if (rows[0] <= rows[1]) {
    for (uint32_t ty = (uint32_t)rows[0] / TILE; ty <= (uint32_t)rows[1] / TILE; ++ty) {
      uint32_t span[2];
      footprint_row_tiles(q, q + 12, q[15], rows, ty, f->image[0], span);
      for (uint32_t x = span[0]; x < span[1]; ++x) {
        if (count < max) out[count] = ty * f->image[2] + x;
        ++count;
      }
    }
  }
  return count;
}

/* Stable counting sort on 16-bit keys: the order RadixSort (radix_sort.cpp:57-83) leaves. */
void gso_depth_order(const uint32_t* keys, uint32_t n, uint32_t* order) {
  uint32_t* count = (uint32_t*)calloc(65537u, sizeof(uint32_t));
  for (uint32_t i = 0; i < n; ++i) ++count[(keys[i] & 0xffffu) + 1u];
  for (uint32_t k = 1; k <= 65536u; ++k) count[k] += count[k - 1];
  for (uint32_t i = 0; i < n; ++i) order[count[keys[i] & 0xffffu]++] = i;
  free(count);
}

uint64_t gso_emit(const gso_frame* f, const float* projected, const uint32_t* tiles, const uint32_t* order,
                  uint32_t n, uint64_t capacity, uint32_t* offsets, uint32_t* pair_tile, uint32_t* pair_gaussian,
                  float* pair_grads, uint32_t* mismatch) {
  /* train_gather.comp:15-18 + exclusive scan (scan_local/blocks/add): offsets in depth order. */
  uint64_t* sorted_offsets = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1u));
  uint64_t total = 0;
  for (uint32_t k = 0; k < n; ++k) {
    sorted_offsets[k] = total;
    total += tiles[order[k]];
  }
  uint32_t bad = 0;
  const uint32_t pad_tile = f->image[2] * f->image[3];
  /* train_emit.comp:26-63 */
  PAR_FOR
  for (int64_t kk = 0; kk < (int64_t)n; ++kk) {
    const uint32_t i = order[kk];
    if (tiles[i] == 0u) continue;
    const float* q = projected + (size_t)i * 16u;
    uint64_t p = sorted_offsets[kk];
    offsets[i] = (uint32_t)p;
    const uint64_t end = p + tiles[i] < capacity ? p + tiles[i] : capacity;
    uint32_t wanted = 0u;
    int rows[2];
    footprint_rows(q, q + 12, q[15], f->image[1], rows);
    if (rows[0] <= rows[1]) {
      for (uint32_t ty = (uint32_t)rows[0] / TILE; ty <= (uint32_t)rows[1] / TILE; ++ty) {
        uint32_t span[2];
        footprint_row_tiles(q, q + 12, q[15], rows, ty, f->image[0], span);
        wanted += span[1] - span[0];
        for (uint32_t x = span[0]; x < span[1] && p < end; ++x) {
          pair_tile[p] = ty * f->image[2] + x;
          pair_gaussian[p] = i;
          ++p;
        }
      }
    }
    if (wanted == tiles[i]) continue;
#pragma omp atomic
    ++bad;
    for (; p < end; ++p) {
      pair_tile[p] = pad_tile;
      pair_gaussian[p] = i;
      if (pair_grads) memset(pair_grads + p * 12u, 0, 12u * sizeof(float));
    }
  }
  free(sorted_offsets);
  if (mismatch) *mismatch = bad;
  return total;
}

void gso_sort_pairs(const uint32_t* pair_tile, uint64_t pairs, uint32_t num_tiles, uint32_t* render_order,
                    uint32_t* sorted_tile, uint32_t* ranges) {
  const uint32_t bins = num_tiles + 1u;
  uint64_t* start = (uint64_t*)calloc(bins + 1u, sizeof(uint64_t));
  for (uint64_t p = 0; p < pairs; ++p) ++start[pair_tile[p] + 1u];
  for (uint32_t t = 1; t <= bins; ++t) start[t] += start[t - 1];
  for (uint32_t t = 0; t < bins; ++t) {
    ranges[2u * t] = (uint32_t)start[t];
    ranges[2u * t + 1u] = (uint32_t)start[t + 1u];
    if (start[t] == start[t + 1u]) ranges[2u * t] = ranges[2u * t + 1u] = 0u; /* cleared to (0, 0) */
  }
  for (uint64_t p = 0; p < pairs; ++p) {
    const uint64_t k = start[pair_tile[p]]++;
    render_order[k] = (uint32_t)p;
    if (sorted_tile) sorted_tile[k] = pair_tile[p];
  }
  free(start);
}

static float pixel_weight(const float head[4], float px, float py) {
  if (head[2] <= 0.0f) return 1.0f;
  const float dx = px - head[0], dy = py - head[1];
  const float d = sqrtf(dx * dx + dy * dy) / head[2];
  const float s = clampf((d - 0.8f) / 0.2f, 0.0f, 1.0f);
  return 1.0f + (head[3] - 1.0f) * (1.0f - s * s * (3.0f - 2.0f * s));
}

static uint32_t pack_unorm(float v) { return (uint32_t)(clampf(v, 0.0f, 1.0f) * 255.0f + 0.5f); }

/* train_forward.comp:59-183 (without bucket state). */
void gso_forward(const gso_frame* f, const float* projected, const uint32_t* ranges, const uint32_t* render_order,
                 const uint32_t* pair_gaussian, const uint32_t* target, float* pixel_grad, uint32_t* pixel_count,
                 uint32_t* image, float* tile_loss, uint32_t* tile_count, float* ssim_input, float* pixel_dot) {
  const uint32_t width = f->image[0], height = f->image[1], tiles_x = f->image[2], tiles_y = f->image[3];
  const uint32_t flags = f->model[3];
  PAR_FOR
  for (int64_t tt = 0; tt < (int64_t)tiles_x * tiles_y; ++tt) {
    const uint32_t tile_id = (uint32_t)tt;
    const uint32_t tx = tile_id % tiles_x, ty = tile_id / tiles_x;
    const uint32_t r0 = ranges[2u * tile_id], r1 = ranges[2u * tile_id + 1u];
    float f_loss[2] = {0, 0}, f_more[4] = {0, 0, 0, 0}, f_rr[4] = {0, 0, 0, 0}, f_rp[4] = {0, 0, 0, 0};
    uint32_t max_last = 0u;
    for (uint32_t lid = 0; lid < TILE * TILE; ++lid) {
      const uint32_t x = tx * TILE + lid % TILE, y = ty * TILE + lid / TILE;
      if (x >= width || y >= height) continue;
      const float cx = (float)x + 0.5f, cy = (float)y + 0.5f;
      float T = 1.0f, C[3] = {0.0f, 0.0f, 0.0f};
      uint32_t contributor = 0u, last = 0u;
      for (uint32_t k = r0; k < r1; ++k) {
        ++contributor;
        const float* q = projected + (size_t)pair_gaussian[render_order[k]] * 16u;
        const float dx = q[0] - cx, dy = q[1] - cy;
        const float power = -0.5f * (q[4] * dx * dx + q[6] * dy * dy) - q[5] * dx * dy;
        if (power > 0.0f) continue;
        const float alpha = fminf(kMaxAlpha, q[3] * expf(power));
        if (alpha < kMinAlpha) continue;
        const float next_T = T * (1.0f - alpha);
        if (next_T < kMinTransmittance) break;
        for (int c = 0; c < 3; ++c) C[c] += q[8 + c] * alpha * T;
        T = next_T;
        last = contributor;
      }
      const size_t pix = (size_t)y * width + x;
      const float* bg = f->background;
      float out[3], tc[3], e[3], dldc[3];
      const uint32_t t = target[pix];
      const float tr[4] = {(float)(t & 255u) / 255.0f, (float)((t >> 8) & 255u) / 255.0f,
                           (float)((t >> 16) & 255u) / 255.0f, (float)(t >> 24) / 255.0f};
      const float w = pixel_weight(f->head, cx, cy);
      for (int c = 0; c < 3; ++c) {
        out[c] = C[c] + T * bg[c];
        const float photo = tr[c] * f->exposure[c];
        tc[c] = (flags & GSO_FLAG_MASKED) ? bg[c] * (1.0f - tr[3]) + photo * tr[3] : photo;
        e[c] = out[c] - tc[c];
        const float sgn = e[c] > 0.0f ? 1.0f : (e[c] < 0.0f ? -1.0f : 0.0f);
        dldc[c] = sgn * ((1.0f - f->loss[0]) * f->background[3] * w);
      }
      if (ssim_input) {
        float* si = ssim_input + pix * 8u;
        si[0] = out[0]; si[1] = out[1]; si[2] = out[2]; si[3] = w;
        si[4] = tc[0]; si[5] = tc[1]; si[6] = tc[2]; si[7] = 0.0f;
      }
      float* pg = pixel_grad + pix * 4u;
      pg[0] = dldc[0]; pg[1] = dldc[1]; pg[2] = dldc[2]; pg[3] = T;
      if (pixel_dot) pixel_dot[pix] = dldc[0] * out[0] + dldc[1] * out[1] + dldc[2] * out[2];
      pixel_count[pix] = last;
      image[pix] = pack_unorm(out[0]) | pack_unorm(out[1]) << 8 | pack_unorm(out[2]) << 16 | pack_unorm(1.0f - T) << 24;
      const float l0 = fabsf(e[0]) + fabsf(e[1]) + fabsf(e[2]);
      const float l1 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
      f_loss[0] += l0;
      f_loss[1] += l1;
      f_more[0] += w * l0;
      f_more[1] += 3.0f * w;
      const float hx = cx - f->head[0], hy = cy - f->head[1];
      if (f->head[2] > 0.0f && sqrtf(hx * hx + hy * hy) <= f->head[2]) {
        f_more[2] += l1;
        f_more[3] += 1.0f;
      }
      if (tr[3] > 0.95f && T < 0.05f) {
        for (int c = 0; c < 3; ++c) {
          f_rr[c] += C[c] * C[c];
          f_rp[c] += C[c] * tr[c];
        }
        f_rr[3] += 1.0f;
      }
      f_rp[3] += tr[3] > 0.0f ? 1.0f : 0.0f;
      if (last > max_last) max_last = last;
    }
    float* tl = tile_loss + (size_t)tile_id * 16u;
    tl[0] = f_loss[0]; tl[1] = f_loss[1]; tl[2] = 0.0f; tl[3] = f_more[0];
    tl[4] = 0.0f; tl[5] = f_more[1]; tl[6] = f_more[2]; tl[7] = f_more[3];
    for (int c = 0; c < 4; ++c) {
      tl[8 + c] = f_rr[c];
      tl[12 + c] = f_rp[c];
    }
    tile_count[tile_id] = max_last;
  }
}

/* Separable 11-tap window (rows, then columns), zero outside the image, as
   train_ssim.comp:70-108 evaluates it per tile with a 5-pixel halo. */
static void blur(const float* in, float* tmp, float* out, uint32_t width, uint32_t height) {
  PAR_FOR
  for (int64_t yy = 0; yy < (int64_t)height; ++yy) {
    for (uint32_t x = 0; x < width; ++x) {
      float s = 0.0f;
      for (int k = 0; k <= 10; ++k) {
        const int xx = (int)x + k - 5;
        const float v = xx >= 0 && xx < (int)width ? in[(size_t)yy * width + (uint32_t)xx] : 0.0f;
        s += kSsimWindow[k] * v;
      }
      tmp[(size_t)yy * width + x] = s;
    }
  }
  PAR_FOR
  for (int64_t yy = 0; yy < (int64_t)height; ++yy) {
    for (uint32_t x = 0; x < width; ++x) {
      float s = 0.0f;
      for (int k = 0; k <= 10; ++k) {
        const int y2 = (int)yy + k - 5;
        const float v = y2 >= 0 && y2 < (int)height ? tmp[(size_t)y2 * width + x] : 0.0f;
        s += kSsimWindow[k] * v;
      }
      out[(size_t)yy * width + x] = s;
    }
  }
}

/* train_ssim.comp:35-47 */
static int background_only(const gso_frame* f, const uint32_t* ranges, const float* tile_loss, int tx, int ty) {
  if ((f->model[3] & GSO_FLAG_MASKED) == 0u) return 0;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      const int nx = tx + dx, ny = ty + dy;
      if (nx < 0 || ny < 0 || nx >= (int)f->image[2] || ny >= (int)f->image[3]) continue;
      const uint32_t t = (uint32_t)ny * f->image[2] + (uint32_t)nx;
      if (ranges[2u * t + 1u] > ranges[2u * t] || tile_loss[t * 16u + 15u] > 0.0f) return 0;
    }
  return 1;
}

void gso_ssim(const gso_frame* f, const float* ssim_input, const uint32_t* ranges, float* ssim_maps,
              float* tile_loss) {
  const uint32_t width = f->image[0], height = f->image[1], tiles_x = f->image[2], tiles_y = f->image[3];
  const size_t n = (size_t)width * height;
  float* in = (float*)malloc(sizeof(float) * n * 5u);
  float* mom = (float*)malloc(sizeof(float) * n * 5u);
  float* tmp = (float*)malloc(sizeof(float) * n);
  float* ssim = (float*)malloc(sizeof(float) * n * 3u);
  const float c1 = f->loss[1], c2 = f->loss[2];
  for (int c = 0; c < 3; ++c) {
    for (size_t p = 0; p < n; ++p) {
      const float x = ssim_input[p * 8u + (size_t)c], y = ssim_input[p * 8u + 4u + (size_t)c];
      in[p] = x;
      in[n + p] = y;
      in[2u * n + p] = x * x;
      in[3u * n + p] = y * y;
      in[4u * n + p] = x * y;
    }
    for (int q = 0; q < 5; ++q) blur(in + (size_t)q * n, tmp, mom + (size_t)q * n, width, height);
    for (size_t p = 0; p < n; ++p) {
      const float mx = mom[p], my = mom[n + p], exx = mom[2u * n + p], eyy = mom[3u * n + p], exy = mom[4u * n + p];
      const float vx = exx - mx * mx, vy = eyy - my * my, cxy = exy - mx * my;
      const float l = 2.0f * mx * my + c1, cs = 2.0f * cxy + c2;
      const float m = mx * mx + my * my + c1, v = vx + vy + c2;
      const float inv = 1.0f / (m * v);
      const float s = l * cs * inv;
      const float d_cxy = 2.0f * l * inv;
      const float d_vx = -s / v;
      const float a = 2.0f * my * cs * inv - s * 2.0f * mx / m - 2.0f * mx * d_vx - my * d_cxy;
      const float w = ssim_input[p * 8u + 3u];
      ssim_maps[p * 9u + (size_t)c] = w * a;
      ssim_maps[p * 9u + 3u + (size_t)c] = w * d_vx;
      ssim_maps[p * 9u + 6u + (size_t)c] = w * d_cxy;
      ssim[p * 3u + (size_t)c] = s;
    }
  }
  for (uint32_t ty = 0; ty < tiles_y; ++ty)
    for (uint32_t tx = 0; tx < tiles_x; ++tx) {
      const uint32_t t = ty * tiles_x + tx;
      float* tl = tile_loss + (size_t)t * 16u;
      if (background_only(f, ranges, tile_loss, (int)tx, (int)ty)) {
        const uint32_t sx = width - tx * TILE < TILE ? width - tx * TILE : TILE;
        const uint32_t sy = height - ty * TILE < TILE ? height - ty * TILE : TILE;
        tl[2] = 3.0f * (float)(sx * sy);
        tl[4] = tl[5];
        continue;
      }
      float sum = 0.0f, wsum = 0.0f;
      for (uint32_t lid = 0; lid < TILE * TILE; ++lid) {
        const uint32_t x = tx * TILE + lid % TILE, y = ty * TILE + lid / TILE;
        if (x >= width || y >= height) continue;
        const size_t p = (size_t)y * width + x;
        const float w = ssim_input[p * 8u + 3u];
        float s_sum = 0.0f, w_sum = 0.0f;
        for (int c = 0; c < 3; ++c) {
          s_sum += ssim[p * 3u + (size_t)c];
          w_sum += w * ssim[p * 3u + (size_t)c];
        }
        sum += s_sum;
        wsum += w_sum;
      }
      tl[2] = sum;
      tl[4] = wsum;
    }
  free(in);
  free(mom);
  free(tmp);
  free(ssim);
}

void gso_ssim_grad(const gso_frame* f, const float* ssim_input, const float* ssim_maps, const uint32_t* ranges,
                   float* pixel_grad, float* pixel_dot) {
  const uint32_t width = f->image[0], height = f->image[1], tiles_x = f->image[2];
  const size_t n = (size_t)width * height;
  float* in = (float*)malloc(sizeof(float) * n);
  float* tmp = (float*)malloc(sizeof(float) * n);
  float* g = (float*)malloc(sizeof(float) * n * 9u);
  for (int q = 0; q < 9; ++q) {
    for (size_t p = 0; p < n; ++p) in[p] = ssim_maps[p * 9u + (size_t)q];
    blur(in, tmp, g + (size_t)q * n, width, height);
  }
  const float scale = f->loss[0] * f->background[3];
  for (size_t p = 0; p < n; ++p) {
    const uint32_t x = (uint32_t)(p % width), y = (uint32_t)(p / width);
    const uint32_t t = (y / TILE) * tiles_x + x / TILE;
    /* train_ssim_grad.comp:26-28 (tiles without splats keep their L1 gradient when the target is masked) */
    if ((f->model[3] & GSO_FLAG_MASKED) && ranges[2u * t + 1u] <= ranges[2u * t]) continue;
    float* pg = pixel_grad + p * 4u;
    float dot = 0.0f;
    for (int c = 0; c < 3; ++c) {
      const float xc = ssim_input[p * 8u + (size_t)c], yc = ssim_input[p * 8u + 4u + (size_t)c];
      const float ds = g[(size_t)c * n + p] + 2.0f * xc * g[(size_t)(3 + c) * n + p] + yc * g[(size_t)(6 + c) * n + p];
      pg[c] -= scale * ds;
    }
    for (int c = 0; c < 3; ++c) dot += pg[c] * ssim_input[p * 8u + (size_t)c];
    if (pixel_dot) pixel_dot[p] = dot;
  }
  free(in);
  free(tmp);
  free(g);
}

typedef struct {
  float T, accum[3], last_alpha, last_color[3];
} pixel_state;

/* train_common.glsl:228-253 */
static void splat_pixel_grad(float dx, float dy, const float con[3], float opacity, const float color[3],
                             const float dL_dC[3], float T_final, float bg_dot, pixel_state* st, float g[12]) {
  memset(g, 0, 12u * sizeof(float));
  const float power = -0.5f * (con[0] * dx * dx + con[2] * dy * dy) - con[1] * dx * dy;
  const float G = expf(power);
  const float raw_alpha = opacity * G;
  const float alpha = fminf(kMaxAlpha, raw_alpha);
  if (power > 0.0f || alpha < kMinAlpha) return;
  st->T = st->T / (1.0f - alpha);
  for (int c = 0; c < 3; ++c) st->accum[c] = st->last_alpha * st->last_color[c] + (1.0f - st->last_alpha) * st->accum[c];
  for (int c = 0; c < 3; ++c) st->last_color[c] = color[c];
  float dL_dalpha =
      ((color[0] - st->accum[0]) * dL_dC[0] + (color[1] - st->accum[1]) * dL_dC[1] + (color[2] - st->accum[2]) * dL_dC[2]) *
      st->T;
  st->last_alpha = alpha;
  dL_dalpha += (-T_final / (1.0f - alpha)) * bg_dot;
  const int clamped = raw_alpha >= kMaxAlpha;
  const float dL_dopacity = clamped ? 0.0f : G * dL_dalpha;
  const float dL_dpower = clamped ? 0.0f : raw_alpha * dL_dalpha;
  const float dmx = dL_dpower * -(con[0] * dx + con[1] * dy);
  const float dmy = dL_dpower * -(con[2] * dy + con[1] * dx);
  g[0] = dmx;
  g[1] = dmy;
  g[2] = dL_dpower * (-0.5f * dx * dx);
  g[3] = dL_dpower * (-dx * dy);
  g[4] = dL_dpower * (-0.5f * dy * dy);
  g[5] = dL_dopacity;
  for (int c = 0; c < 3; ++c) g[6 + c] = (alpha * st->T) * dL_dC[c];
  g[9] = fabsf(dmx);
  g[10] = fabsf(dmy);
  g[11] = 0.0f;
}

void gso_backward(const gso_frame* f, const float* projected, const uint32_t* ranges, const uint32_t* render_order,
                  const uint32_t* pair_gaussian, const float* pixel_grad, const uint32_t* pixel_count,
                  const uint32_t* tile_count, float* pair_grads) {
  const uint32_t width = f->image[0], height = f->image[1], tiles_x = f->image[2], tiles_y = f->image[3];
  PAR_FOR
  for (int64_t tt = 0; tt < (int64_t)tiles_x * tiles_y; ++tt) {
    const uint32_t t = (uint32_t)tt;
    const uint32_t tx = t % tiles_x, ty = t / tiles_x;
    const uint32_t r0 = ranges[2u * t], r1 = ranges[2u * t + 1u];
    uint32_t n = r1 - r0;
    if (tile_count[t] < n) n = tile_count[t];
    for (uint32_t k = r0 + n; k < r1; ++k) memset(pair_grads + (size_t)render_order[k] * 12u, 0, 12u * sizeof(float));
    if (n == 0u) continue;
    pixel_state st[TILE * TILE];
    float dldc[TILE * TILE][3], tfin[TILE * TILE], bgd[TILE * TILE];
    uint32_t last[TILE * TILE];
    int inside[TILE * TILE];
    for (uint32_t lid = 0; lid < TILE * TILE; ++lid) {
      const uint32_t x = tx * TILE + lid % TILE, y = ty * TILE + lid / TILE;
      inside[lid] = x < width && y < height;
      const size_t pix = (size_t)y * width + x;
      for (int c = 0; c < 3; ++c) dldc[lid][c] = inside[lid] ? pixel_grad[pix * 4u + (size_t)c] : 0.0f;
      tfin[lid] = inside[lid] ? pixel_grad[pix * 4u + 3u] : 0.0f;
      last[lid] = inside[lid] ? pixel_count[pix] : 0u;
      bgd[lid] = f->background[0] * dldc[lid][0] + f->background[1] * dldc[lid][1] + f->background[2] * dldc[lid][2];
      memset(&st[lid], 0, sizeof(pixel_state));
      st[lid].T = tfin[lid];
    }
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t pre = render_order[r0 + n - 1u - i];
      const float* q = projected + (size_t)pair_gaussian[pre] * 16u;
      float red[TILE * TILE][12];
      for (uint32_t lid = 0; lid < TILE * TILE; ++lid) {
        memset(red[lid], 0, sizeof(red[lid]));
        if (inside[lid] && n - i <= last[lid]) {
          const float cx = (float)(tx * TILE + lid % TILE) + 0.5f, cy = (float)(ty * TILE + lid / TILE) + 0.5f;
          splat_pixel_grad(q[0] - cx, q[1] - cy, q + 4, q[3], q + 8, dldc[lid], tfin[lid], bgd[lid], &st[lid], red[lid]);
        }
      }
      float rows[TILE][12];
      for (uint32_t r = 0; r < TILE; ++r) {
        for (int c = 0; c < 12; ++c) rows[r][c] = 0.0f;
        for (uint32_t x = 0; x < TILE; ++x)
          for (int c = 0; c < 12; ++c) rows[r][c] += red[r * TILE + x][c];
      }
      float* out = pair_grads + (size_t)pre * 12u;
      for (int c = 0; c < 12; ++c) out[c] = 0.0f;
      for (uint32_t r = 0; r < TILE; ++r)
        for (int c = 0; c < 12; ++c) out[c] += rows[r][c];
    }
  }
}

void gso_pair_sum(uint32_t n, const uint32_t* tiles, const uint32_t* offsets, const float* pair_grads,
                  float* grad_sum) {
  PAR_FOR
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    float a[12] = {0};
    if (tiles[ii] > 0u) {
      const size_t first = offsets[ii];
      for (uint32_t k = 0; k < tiles[ii]; ++k)
        for (int c = 0; c < 12; ++c) a[c] += pair_grads[(first + k) * 12u + (size_t)c];
    }
    memcpy(grad_sum + (size_t)ii * 12u, a, sizeof(a));
  }
}

/* train_step.glsl:72-220 (no pose or motion). */
void gso_project_backward(const gso_frame* f, const float* params, const float* sh, const uint32_t* tiles,
                          const float* grad_sum, const float* projected, float* stats, float* grad16,
                          float* sh_input, uint8_t* drew_out) {
  const uint32_t n = f->model[0];
  PAR_FOR
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const uint32_t i = (uint32_t)ii;
    const float* pp = params + (size_t)i * 16u;
    float* si = sh_input + (size_t)i * 8u;
    if (pp[7] < 0.5f) continue;
    for (int k = 0; k < 8; ++k) si[k] = 0.0f;
    if (tiles[i] == 0u) continue;
    const float* a = grad_sum + (size_t)i * 12u;
    int drew = 0;
    for (int k = 0; k < 12; ++k) drew |= a[k] != 0.0f;
    if (drew_out && drew) drew_out[i] |= 1u;
    const float dL_dmean[2] = {a[0], a[1]};
    const float dL_dconic[3] = {a[2], a[3], a[4]};
    const float dL_dopacity = a[5];
    float dL_dcolor[3] = {a[6], a[7], a[8]};
    const float width = (float)f->image[0], height = (float)f->image[1];
    const float ndc[2] = {0.5f * width, 0.5f * height};
    float* st = stats + (size_t)i * 4u;
    {
      const float gx = dL_dmean[0] * ndc[0], gy = dL_dmean[1] * ndc[1];
      st[0] += sqrtf(gx * gx + gy * gy);
      st[1] += 1.0f;
      st[2] = fmaxf(st[2], projected[(size_t)i * 16u + 7u]);
      const float ax = a[9] * ndc[0], ay = a[10] * ndc[1];
      st[3] += sqrtf(ax * ax + ay * ay);
    }
    const float pos[3] = {pp[0], pp[1], pp[2]};
    float t[3];
    for (int r = 0; r < 3; ++r) t[r] = f->rot[r][0] * pos[0] + f->rot[r][1] * pos[1] + f->rot[r][2] * pos[2] + f->rot[r][3];
    const float fx = f->intrinsics[0], fy = f->intrinsics[1], cx = f->intrinsics[2], cy = f->intrinsics[3];
    const float inv_z = 1.0f / t[2];
    const float lim_x = 1.3f * fmaxf(cx, width - cx) / fx;
    const float lim_y = 1.3f * fmaxf(cy, height - cy) / fy;
    const float rx = t[0] * inv_z, ry = t[1] * inv_z;
    const int clamp_x = rx < -lim_x || rx > lim_x;
    const int clamp_y = ry < -lim_y || ry > lim_y;
    const float tx = clampf(rx, -lim_x, lim_x), ty = clampf(ry, -lim_y, lim_y);
    /* J[row][col] */
    float J[3][3] = {{fx * inv_z, 0.0f, -fx * tx * inv_z}, {0.0f, fy * inv_z, -fy * ty * inv_z}, {0, 0, 0}};
    const float* q = pp + 8;
    const float qlen = fmaxf(sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), 1e-12f);
    const float qn[4] = {q[0] / qlen, q[1] / qlen, q[2] / qlen, q[3] / qlen};
    float R[3][3];
    quat_to_matrix(qn, R);
    const float s[3] = {expf(pp[4]), expf(pp[5]), expf(pp[6])};
    float M[3][3], Sigma[3][3], W[3][3], T[3][3], cov[3][3], tmp[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        M[r][c] = R[r][c] * s[c];
        W[r][c] = f->rot[r][c];
      }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) Sigma[r][c] = M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) T[r][c] = J[r][0] * W[0][c] + J[r][1] * W[1][c] + J[r][2] * W[2][c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) tmp[r][c] = T[r][0] * Sigma[0][c] + T[r][1] * Sigma[1][c] + T[r][2] * Sigma[2][c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) cov[r][c] = tmp[r][0] * T[c][0] + tmp[r][1] * T[c][1] + tmp[r][2] * T[c][2];
    const float A = cov[0][0] + kDilation, B = cov[1][0], C = cov[1][1] + kDilation;
    const float D = A * C - B * B;

    /* Colour -> SH and view direction. */
    float dir_raw[3] = {pos[0] - f->cam_pos[0], pos[1] - f->cam_pos[1], pos[2] - f->cam_pos[2]};
    const float dir_len = fmaxf(sqrtf(dir_raw[0] * dir_raw[0] + dir_raw[1] * dir_raw[1] + dir_raw[2] * dir_raw[2]), 1e-12f);
    const float dir[3] = {dir_raw[0] / dir_len, dir_raw[1] / dir_len, dir_raw[2] / dir_len};
    uint32_t clamped;
    memcpy(&clamped, &projected[(size_t)i * 16u + 11u], 4);
    for (int c = 0; c < 3; ++c)
      if (clamped & (1u << c)) dL_dcolor[c] = 0.0f;
    const uint32_t degree = f->model[1];
    float basis[16];
    sh_basis(dir, degree, basis);
    float* g16 = grad16 + (size_t)i * 16u;
    for (int c = 0; c < 3; ++c) g16[12 + c] += basis[0] * dL_dcolor[c];
    if (drew_out && (dL_dcolor[0] != 0.0f || dL_dcolor[1] != 0.0f || dL_dcolor[2] != 0.0f)) drew_out[i] |= 2u;
    si[0] = dL_dcolor[0]; si[1] = dL_dcolor[1]; si[2] = dL_dcolor[2]; si[3] = 0.0f;
    si[4] = dir[0]; si[5] = dir[1]; si[6] = dir[2]; si[7] = 0.0f;
    float dL_ddir[3] = {0.0f, 0.0f, 0.0f};
    const int coeffs = sh_rest_coeffs(degree);
    if (coeffs > 0) {
      float db[16][3];
      sh_basis_grad(dir, degree, db);
      const float* shp = sh + (size_t)i * f->model[2];
      for (int k = 0; k < coeffs; ++k) {
        const float w = shp[k * 3] * dL_dcolor[0] + shp[k * 3 + 1] * dL_dcolor[1] + shp[k * 3 + 2] * dL_dcolor[2];
        for (int ax = 0; ax < 3; ++ax) dL_ddir[ax] += w * db[k + 1][ax];
      }
    }
    const float ddot = dir[0] * dL_ddir[0] + dir[1] * dL_ddir[1] + dir[2] * dL_ddir[2];
    float dL_ddir_raw[3];
    for (int ax = 0; ax < 3; ++ax) dL_ddir_raw[ax] = (dL_ddir[ax] - dir[ax] * ddot) / dir_len;

    /* Opacity. */
    const float opacity = sigmoidf(pp[3]);
    g16[3] += dL_dopacity * opacity * (1.0f - opacity);

    /* Conic -> dilated 2D covariance. */
    const float ga = dL_dconic[0], gb = dL_dconic[1], gc = dL_dconic[2];
    const float inv_d2 = 1.0f / (D * D);
    const float gA = (-C * C * ga + B * C * gb - B * B * gc) * inv_d2;
    const float gB = (2.0f * B * C * ga - (D + 2.0f * B * B) * gb + 2.0f * A * B * gc) * inv_d2;
    const float gC = (-B * B * ga + A * B * gb - A * A * gc) * inv_d2;
    const float G2[3][3] = {{gA, 0.5f * gB, 0.0f}, {0.5f * gB, gC, 0.0f}, {0.0f, 0.0f, 0.0f}};

    /* dSigma = T^T G2 T, dT = 2 G2 T Sigma, dJ = dT W^T */
    float dSigma[3][3], dT[3][3], dJ[3][3], G2T[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) G2T[r][c] = G2[r][0] * T[0][c] + G2[r][1] * T[1][c] + G2[r][2] * T[2][c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) dSigma[r][c] = T[0][r] * G2T[0][c] + T[1][r] * G2T[1][c] + T[2][r] * G2T[2][c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        dT[r][c] = 2.0f * (G2T[r][0] * Sigma[0][c] + G2T[r][1] * Sigma[1][c] + G2T[r][2] * Sigma[2][c]);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) dJ[r][c] = dT[r][0] * W[c][0] + dT[r][1] * W[c][1] + dT[r][2] * W[c][2];
    /* GLSL dJ[col][row]: dJ[0][0] -> (0,0), dJ[1][1] -> (1,1), dJ[2][0] -> row 0 col 2, dJ[2][1] -> row 1 col 2 */
    float dL_dt[3] = {0.0f, 0.0f, 0.0f};
    const float inv_z2 = inv_z * inv_z;
    dL_dt[2] += -fx * inv_z2 * dJ[0][0] - fy * inv_z2 * dJ[1][1];
    if (clamp_x) {
      dL_dt[2] += fx * tx * inv_z2 * dJ[0][2];
    } else {
      dL_dt[0] += -fx * inv_z2 * dJ[0][2];
      dL_dt[2] += 2.0f * fx * t[0] * inv_z2 * inv_z * dJ[0][2];
    }
    if (clamp_y) {
      dL_dt[2] += fy * ty * inv_z2 * dJ[1][2];
    } else {
      dL_dt[1] += -fy * inv_z2 * dJ[1][2];
      dL_dt[2] += 2.0f * fy * t[1] * inv_z2 * inv_z * dJ[1][2];
    }
    dL_dt[0] += dL_dmean[0] * fx * inv_z;
    dL_dt[1] += dL_dmean[1] * fy * inv_z;
    dL_dt[2] += -(dL_dmean[0] * fx * t[0] + dL_dmean[1] * fy * t[1]) * inv_z2;
    /* dL/dx = W^T dL_dt + dL_ddir_raw */
    for (int c = 0; c < 3; ++c)
      g16[c] += W[0][c] * dL_dt[0] + W[1][c] * dL_dt[1] + W[2][c] * dL_dt[2] + dL_ddir_raw[c];

    /* 3D covariance -> scale, rotation. dM = 2 dSigma M */
    float dM[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) dM[r][c] = 2.0f * (dSigma[r][0] * M[0][c] + dSigma[r][1] * M[1][c] + dSigma[r][2] * M[2][c]);
    for (int c = 0; c < 3; ++c) g16[4 + c] += (dM[0][c] * R[0][c] + dM[1][c] * R[1][c] + dM[2][c] * R[2][c]) * s[c];
    float g[3][3]; /* g[r][c] = dL/dR[r][c] */
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) g[r][c] = dM[r][c] * s[c];
    const float w = qn[0], x = qn[1], y = qn[2], z = qn[3];
    float dqn[4];
    dqn[0] = 2.0f * (-z * g[0][1] + y * g[0][2] + z * g[1][0] - x * g[1][2] - y * g[2][0] + x * g[2][1]);
    dqn[1] = 2.0f * (y * g[0][1] + z * g[0][2] + y * g[1][0] - 2.0f * x * g[1][1] - w * g[1][2] + z * g[2][0] + w * g[2][1] -
                     2.0f * x * g[2][2]);
    dqn[2] = 2.0f * (-2.0f * y * g[0][0] + x * g[0][1] + w * g[0][2] + x * g[1][0] + z * g[1][2] - w * g[2][0] + z * g[2][1] -
                     2.0f * y * g[2][2]);
    dqn[3] = 2.0f * (-2.0f * z * g[0][0] - w * g[0][1] + x * g[0][2] + w * g[1][0] - 2.0f * z * g[1][1] + y * g[1][2] +
                     x * g[2][0] + y * g[2][1]);
    const float qd = qn[0] * dqn[0] + qn[1] * dqn[1] + qn[2] * dqn[2] + qn[3] * dqn[3];
    for (int k = 0; k < 4; ++k) g16[8 + k] += (dqn[k] - qn[k] * qd) / qlen;
  }
}

void gso_sh_gradient(const gso_frame* f, const float* params, const float* sh_input, float* grad_sh) {
  const uint32_t n = f->model[0], stride = f->model[2], degree = f->model[1];
  const int coeffs = sh_rest_coeffs(degree);
  if (coeffs == 0) return;
  PAR_FOR
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const size_t i = (size_t)ii;
    if (params[i * 16u + 7u] < 0.5f) continue;
    const float* si = sh_input + i * 8u;
    float basis[16];
    sh_basis(si + 4, degree, basis);
    for (int k = 0; k < coeffs; ++k)
      for (int c = 0; c < 3; ++c) grad_sh[i * stride + (size_t)(k * 3 + c)] += basis[k + 1] * si[c];
  }
}

static float adam1(float p, float g, float* m, float* v, float lr, const gso_frame* f) {
  const float b1 = f->adam[0], b2 = f->adam[1];
  const float mn = g * (1.0f - b1) + *m * b1;
  const float vn = g * g * (1.0f - b2) + *v * b2;
  *m = mn;
  *v = vn;
  return p - lr * (mn * f->bias[0]) / (sqrtf(vn * f->bias[1]) + f->adam[2]);
}

void gso_adam(const gso_frame* f, float* params, float* sh, float* m, float* v, float* m_sh, float* v_sh,
              const float* grad16, const float* grad_sh, const uint8_t* drew) {
  const uint32_t n = f->model[0], stride = f->model[2], degree = f->model[1];
  const int coeffs = sh_rest_coeffs(degree);
  const int sparse = (f->model[3] & GSO_FLAG_SPARSE_ADAM) != 0u;
  const float lr[16] = {f->lr0[0], f->lr0[0], f->lr0[0], f->lr0[3], f->lr0[1], f->lr0[1], f->lr0[1], 0.0f,
                        f->lr0[2], f->lr0[2], f->lr0[2], f->lr0[2], f->lr1[0], f->lr1[0], f->lr1[0], 0.0f};
  PAR_FOR
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const size_t i = (size_t)ii;
    float* p = params + i * 16u;
    if (p[7] < 0.5f) continue;
    const uint8_t d = drew ? drew[i] : 0u;
    if (!sparse || (d & 1u))
      for (int k = 0; k < 16; ++k)
        p[k] = adam1(p[k], grad16[i * 16u + (size_t)k], &m[i * 16u + (size_t)k], &v[i * 16u + (size_t)k], lr[k], f);
    /* train_step_sh.comp:34-35: the SH step skips on a zero colour gradient */
    if (sparse && !(d & 2u)) continue;
    for (int k = 0; k < coeffs * 3; ++k) {
      const size_t o = i * stride + (size_t)k;
      sh[o] = adam1(sh[o], grad_sh[o], &m_sh[o], &v_sh[o], f->lr1[1], f);
    }
  }
}

void gso_densify_mark(const gso_frame* f, float* params, float* sh, float* m, float* v, float* m_sh, float* v_sh,
                      const float* stats, uint32_t* spawn, uint32_t* free_list, uint32_t* counters) {
  const uint32_t n = f->model[0], stride = f->model[2];
  uint32_t free_count = 0u, pruned = 0u;
  for (uint32_t i = 0; i < n; ++i) {
    float* p = params + (size_t)i * 16u;
    uint32_t action = 0u;
    int release = p[7] < 0.5f;
    if (!release) {
      const float* st = stats + (size_t)i * 4u;
      const float max_scale = expf(fmaxf(p[4], fmaxf(p[5], p[6])));
      int prune = sigmoidf(p[3]) < f->densify0[2];
      if (f->densify0[3] > 0.0f && max_scale > f->densify0[3]) prune = 1;
      if (f->densify1[0] > 0.0f && st[2] > f->densify1[0]) prune = 1;
      if (prune) {
        release = 1;
        ++pruned;
        const float cleared[16] = {0, 0, 0, -20.0f, 0, 0, 0, 0, 1.0f, 0, 0, 0, 0, 0, 0, 0};
        memcpy(p, cleared, sizeof(cleared));
        memset(m + (size_t)i * 16u, 0, 16u * sizeof(float));
        memset(v + (size_t)i * 16u, 0, 16u * sizeof(float));
        for (uint32_t k = 0; k < stride; ++k) {
          sh[(size_t)i * stride + k] = 0.0f;
          m_sh[(size_t)i * stride + k] = 0.0f;
          v_sh[(size_t)i * stride + k] = 0.0f;
        }
      } else if (st[1] > 0.0f && st[0] / st[1] >= f->densify0[0]) {
        action = max_scale <= f->densify0[1] ? 1u : 2u;
      }
    }
    if (release) free_list[free_count++] = i;
    spawn[i] = action;
  }
  counters[0] = free_count;
  counters[2] = pruned;
}

static void clear_state(float* m, float* v, float* m_sh, float* v_sh, uint32_t slot, uint32_t stride) {
  memset(m + (size_t)slot * 16u, 0, 16u * sizeof(float));
  memset(v + (size_t)slot * 16u, 0, 16u * sizeof(float));
  for (uint32_t k = 0; k < stride; ++k) {
    m_sh[(size_t)slot * stride + k] = 0.0f;
    v_sh[(size_t)slot * stride + k] = 0.0f;
  }
}

void gso_densify_spawn(const gso_frame* f, float* params, float* sh, float* m, float* v, float* m_sh, float* v_sh,
                       const uint32_t* spawn, const uint32_t* free_list, uint32_t* counters, uint32_t capacity) {
  const uint32_t n = f->model[0], stride = f->model[2];
  const uint32_t free_count = counters[0];
  uint32_t k = 0u;
  uint32_t seed_bits;
  memcpy(&seed_bits, &f->densify1[1], 4);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t action = spawn[i];
    if (action == 0u) continue;
    const uint32_t kk = k++;
    const uint32_t target = kk < free_count ? free_list[kk] : n + (kk - free_count);
    if (target >= capacity) continue;
    float* p = params + (size_t)i * 16u;
    float p0[4], p1[4], q[4], p3[4];
    memcpy(p0, p, 16);
    memcpy(p1, p + 4, 16);
    memcpy(q, p + 8, 16);
    memcpy(p3, p + 12, 16);
    for (uint32_t c = 0; c < stride; ++c) sh[(size_t)target * stride + c] = sh[(size_t)i * stride + c];
    clear_state(m, v, m_sh, v_sh, target, stride);
    float* t = params + (size_t)target * 16u;
    if (action == 1u) {
      memcpy(t, p0, 16);
      memcpy(t + 4, p1, 16);
    } else {
      uint32_t rng = gso_pcg_hash(i ^ gso_pcg_hash(seed_bits));
      const float s[3] = {expf(p1[0]), expf(p1[1]), expf(p1[2])};
      const float qlen = fmaxf(sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]), 1e-12f);
      const float qn[4] = {q[0] / qlen, q[1] / qlen, q[2] / qlen, q[3] / qlen};
      float R[3][3];
      quat_to_matrix(qn, R);
      float na[3], nb[3];
      normal3(&rng, na);
      normal3(&rng, nb);
      float a[3], b[3];
      for (int r = 0; r < 3; ++r) {
        a[r] = p0[r] + (R[r][0] * (na[0] * s[0]) + R[r][1] * (na[1] * s[1]) + R[r][2] * (na[2] * s[2]));
        b[r] = p0[r] + (R[r][0] * (nb[0] * s[0]) + R[r][1] * (nb[1] * s[1]) + R[r][2] * (nb[2] * s[2]));
      }
      const float ls = logf(f->densify1[2]);
      const float log_scale[3] = {p1[0] - ls, p1[1] - ls, p1[2] - ls};
      p[0] = a[0]; p[1] = a[1]; p[2] = a[2]; p[3] = p0[3];
      p[4] = log_scale[0]; p[5] = log_scale[1]; p[6] = log_scale[2]; p[7] = 1.0f;
      t[0] = b[0]; t[1] = b[1]; t[2] = b[2]; t[3] = p0[3];
      t[4] = log_scale[0]; t[5] = log_scale[1]; t[6] = log_scale[2]; t[7] = 1.0f;
      clear_state(m, v, m_sh, v_sh, i, stride);
    }
    memcpy(t + 8, q, 16);
    memcpy(t + 12, p3, 16);
  }
  counters[1] = k;
}

void gso_reset_opacity(const gso_frame* f, float* params, float* m, float* v, float max_logit) {
  for (uint32_t i = 0; i < f->model[0]; ++i) {
    float* p = params + (size_t)i * 16u;
    if (p[7] < 0.5f) continue;
    p[3] = fminf(p[3], max_logit);
    m[(size_t)i * 16u + 3u] = 0.0f;
    v[(size_t)i * 16u + 3u] = 0.0f;
  }
}

/* ---- FP64 reference forward + loss: train_selftest.cpp:79-283 ---- */

typedef struct {
  int visible;
  double mx, my, depth, opacity, con[3], color[3];
  uint32_t key;
} ref_splat;

static void quat_to_matrix_d(const double q[4], double R[3][3]) {
  const double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const double w = q[0] / n, x = q[1] / n, y = q[2] / n, z = q[3] / n;
  R[0][0] = 1 - 2 * (y * y + z * z);
  R[0][1] = 2 * (x * y - w * z);
  R[0][2] = 2 * (x * z + w * y);
  R[1][0] = 2 * (x * y + w * z);
  R[1][1] = 1 - 2 * (x * x + z * z);
  R[1][2] = 2 * (y * z - w * x);
  R[2][0] = 2 * (x * z - w * y);
  R[2][1] = 2 * (y * z + w * x);
  R[2][2] = 1 - 2 * (x * x + y * y);
}

static void sh_basis_d(const double d[3], int degree, double b[16]) {
  const double x = d[0], y = d[1], z = d[2];
  for (int k = 0; k < 16; ++k) b[k] = 0.0;
  b[0] = 0.28209479177387814;
  if (degree >= 1) {
    b[1] = -0.4886025119029199 * y;
    b[2] = 0.4886025119029199 * z;
    b[3] = -0.4886025119029199 * x;
  }
  if (degree >= 2) {
    const double xx = x * x, yy = y * y, zz = z * z;
    b[4] = 1.0925484305920792 * x * y;
    b[5] = -1.0925484305920792 * y * z;
    b[6] = 0.31539156525252005 * (2 * zz - xx - yy);
    b[7] = -1.0925484305920792 * x * z;
    b[8] = 0.5462742152960396 * (xx - yy);
    if (degree >= 3) {
      b[9] = -0.5900435899266435 * y * (3 * xx - yy);
      b[10] = 2.890611442640554 * x * y * z;
      b[11] = -0.4570457994644658 * y * (4 * zz - xx - yy);
      b[12] = 0.3731763325901154 * z * (2 * zz - 3 * xx - 3 * yy);
      b[13] = -0.4570457994644658 * x * (4 * zz - xx - yy);
      b[14] = 1.445305721320277 * z * (xx - yy);
      b[15] = -0.5900435899266435 * x * (xx - 3 * yy);
    }
  }
}

/* train_selftest.cpp:79-150 */
static ref_splat project_d(const double* cam, uint32_t width, uint32_t height, const double* p, const double* sh,
                           int degree) {
  ref_splat r;
  memset(&r, 0, sizeof(r));
  const double* rot = cam;
  const double* trans = cam + 9;
  const double* position = cam + 12;
  double t[3];
  for (int k = 0; k < 3; ++k) {
    t[k] = trans[k];
    for (int c = 0; c < 3; ++c) t[k] += rot[k * 3 + c] * p[c];
  }
  const double opacity = 1.0 / (1.0 + exp(-p[3]));
  if (p[7] < 0.5 || t[2] <= 0.02 || opacity < 1.0 / 255.0) return r;
  const double fx = cam[15], fy = cam[16], cx = cam[17], cy = cam[18], W = width, H = height;
  const double z = t[2];
  const double lim_x = 1.3 * fmax(cx, W - cx) / fx, lim_y = 1.3 * fmax(cy, H - cy) / fy;
  const double tx = fmin(fmax(t[0] / z, -lim_x), lim_x), ty = fmin(fmax(t[1] / z, -lim_y), lim_y);
  const double J[2][3] = {{fx / z, 0, -fx * tx / z}, {0, fy / z, -fy * ty / z}};
  double R[3][3];
  quat_to_matrix_d(p + 8, R);
  double M[3][3], Sigma[3][3], T[2][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) M[a][b] = R[a][b] * exp(p[4 + b]);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      Sigma[a][b] = 0;
      for (int k = 0; k < 3; ++k) Sigma[a][b] += M[a][k] * M[b][k];
    }
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 3; ++b) {
      T[a][b] = 0;
      for (int k = 0; k < 3; ++k) T[a][b] += J[a][k] * rot[k * 3 + b];
    }
  double cov[2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      cov[a][b] = 0;
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) cov[a][b] += T[a][k] * Sigma[k][l] * T[b][l];
    }
  const double A = cov[0][0] + 0.3, B = cov[0][1], C = cov[1][1] + 0.3;
  const double det = A * C - B * B;
  if (det <= 0) return r;
  r.visible = 1;
  r.mx = fx * t[0] / z + cx;
  r.my = fy * t[1] / z + cy;
  r.depth = z;
  r.opacity = opacity;
  r.con[0] = C / det;
  r.con[1] = -B / det;
  r.con[2] = A / det;
  double dir[3], len = 0;
  for (int k = 0; k < 3; ++k) {
    dir[k] = p[k] - position[k];
    len += dir[k] * dir[k];
  }
  len = sqrt(len);
  for (int k = 0; k < 3; ++k) dir[k] /= len;
  double b[16];
  sh_basis_d(dir, degree, b);
  const int coeffs = degree == 0 ? 0 : (degree + 1) * (degree + 1) - 1;
  for (int c = 0; c < 3; ++c) {
    double v = b[0] * p[12 + c];
    for (int k = 0; k < coeffs; ++k) v += b[k + 1] * sh[k * 3 + c];
    r.color[c] = fmax(v + 0.5, 0.0);
  }
  const double kq = log2(z / 0.02) / log2(1000.0 / 0.02);
  r.key = (uint32_t)(fmin(fmax(kq, 0.0), 1.0) * 65535.0);
  return r;
}

double gso_reference_ssim(const double* x, const double* y, uint32_t width, uint32_t height, const double* weights) {
  const int R = 5;
  double w[11], total = 0.0;
  for (int k = -R; k <= R; ++k) total += w[k + R] = exp(-(double)(k * k) / (2.0 * 1.5 * 1.5));
  for (int k = 0; k < 11; ++k) w[k] /= total;
  const double c1 = 0.01 * 0.01, c2 = 0.03 * 0.03;
  const size_t n = (size_t)width * height;
  double* in = (double*)malloc(sizeof(double) * n * 5u);
  double* rows = (double*)calloc(n * 5u, sizeof(double));
  double* out = (double*)calloc(n * 5u, sizeof(double));
  double sum = 0.0;
  for (int c = 0; c < 3; ++c) {
    for (size_t p = 0; p < n; ++p) {
      const double a = x[p * 3 + (size_t)c], b = y[p * 3 + (size_t)c];
      const double v[5] = {a, b, a * a, b * b, a * b};
      for (int q = 0; q < 5; ++q) in[(size_t)q * n + p] = v[q];
    }
    for (int q = 0; q < 5; ++q) {
      for (uint32_t r = 0; r < height; ++r)
        for (uint32_t col = 0; col < width; ++col) {
          double s = 0.0;
          for (int k = -R; k <= R; ++k) {
            const int cc = (int)col + k;
            if (cc >= 0 && cc < (int)width) s += w[k + R] * in[(size_t)q * n + (size_t)r * width + (size_t)cc];
          }
          rows[(size_t)q * n + (size_t)r * width + col] = s;
        }
      for (uint32_t r = 0; r < height; ++r)
        for (uint32_t col = 0; col < width; ++col) {
          double s = 0.0;
          for (int k = -R; k <= R; ++k) {
            const int rr = (int)r + k;
            if (rr >= 0 && rr < (int)height) s += w[k + R] * rows[(size_t)q * n + (size_t)rr * width + col];
          }
          out[(size_t)q * n + (size_t)r * width + col] = s;
        }
    }
    for (size_t p = 0; p < n; ++p) {
      const double mx = out[p], my = out[n + p];
      const double vx = out[2 * n + p] - mx * mx, vy = out[3 * n + p] - my * my, cxy = out[4 * n + p] - mx * my;
      const double wt = weights ? weights[p] : 1.0;
      sum += wt * (2 * mx * my + c1) * (2 * cxy + c2) / ((mx * mx + my * my + c1) * (vx + vy + c2));
    }
  }
  free(in);
  free(rows);
  free(out);
  return sum / (3.0 * (double)n);
}

typedef struct {
  const ref_splat* refs;
} sort_ctx;

double gso_reference_loss(const double* camera, uint32_t width, uint32_t height, const double* params,
                          const double* sh, uint32_t n, int stride, int degree, const uint8_t* target,
                          const float* bg, int masked, double lambda, double* image, const double* head,
                          uint64_t* signature) {
  uint64_t sig = 1469598103934665603ull; /* FNV-1a over every blend decision */
  const size_t pixels = (size_t)width * height;
  double* render = (double*)malloc(sizeof(double) * pixels * 3u);
  double* truth = (double*)malloc(sizeof(double) * pixels * 3u);
  double* weights = (double*)malloc(sizeof(double) * pixels);
  ref_splat* refs = (ref_splat*)malloc(sizeof(ref_splat) * (n > 0 ? n : 1));
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n > 0 ? n : 1));
  for (uint32_t i = 0; i < n; ++i) refs[i] = project_d(camera, width, height, params + (size_t)i * 16u, sh + (size_t)i * (size_t)stride, degree);
  /* std::stable_sort by key: a stable counting sort gives the same order. */
  uint32_t count = 0;
  {
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (n > 0 ? n : 1));
    uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * (n > 0 ? n : 1));
    for (uint32_t i = 0; i < n; ++i)
      if (refs[i].visible) {
        keys[count] = refs[i].key;
        idx[count++] = i;
      }
    uint32_t* o = (uint32_t*)malloc(sizeof(uint32_t) * (count > 0 ? count : 1));
    gso_depth_order(keys, count, o);
    for (uint32_t k = 0; k < count; ++k) order[k] = idx[o[k]];
    free(o);
    free(keys);
    free(idx);
  }
  double weighted_l1 = 0.0, weight_sum = 0.0;
  for (uint32_t y = 0; y < height; ++y)
    for (uint32_t x = 0; x < width; ++x) {
      double T = 1, C[3] = {0, 0, 0};
      for (uint32_t k = 0; k < count; ++k) {
        const ref_splat* g = &refs[order[k]];
        const double dx = g->mx - (x + 0.5), dy = g->my - (y + 0.5);
        const double power = -0.5 * (g->con[0] * dx * dx + g->con[2] * dy * dy) - g->con[1] * dx * dy;
        if (power > 0) continue;
        const double raw = g->opacity * exp(power);
        const double alpha = fmin(0.99, raw);
        if (alpha < 1.0 / 255.0) continue;
        if (T * (1 - alpha) < 1e-4) {
          sig = (sig ^ (0x100000000ull | order[k])) * 1099511628211ull;
          break;
        }
        sig = (sig ^ ((raw >= 0.99 ? 0x200000000ull : 0ull) | order[k])) * 1099511628211ull;
        for (int c = 0; c < 3; ++c) C[c] += g->color[c] * alpha * T;
        T *= 1 - alpha;
      }
      sig = (sig ^ 0xffffffffffull) * 1099511628211ull; /* pixel boundary */
      const uint8_t* t = &target[((size_t)y * width + x) * 4u];
      const double a = t[3] / 255.0;
      for (int c = 0; c < 3; ++c) {
        const double out = C[c] + T * bg[c];
        const double tc = masked ? bg[c] * (1 - a) + t[c] / 255.0 * a : t[c] / 255.0;
        render[((size_t)y * width + x) * 3u + (size_t)c] = out;
        truth[((size_t)y * width + x) * 3u + (size_t)c] = tc;
      }
      double w = 1.0;
      if (head != NULL && head[2] > 0.0) {
        const double d = hypot(x + 0.5 - head[0], y + 0.5 - head[1]) / head[2];
        const double s = fmin(fmax((d - 0.8) / 0.2, 0.0), 1.0);
        w = 1.0 + (head[3] - 1.0) * (1.0 - s * s * (3.0 - 2.0 * s));
      }
      weights[(size_t)y * width + x] = w;
      for (int c = 0; c < 3; ++c) {
        const size_t i = ((size_t)y * width + x) * 3u + (size_t)c;
        weighted_l1 += w * fabs(render[i] - truth[i]);
      }
      weight_sum += 3.0 * w;
    }
  if (image) memcpy(image, render, sizeof(double) * pixels * 3u);
  if (signature) {
    /* Depth order and colour clamps change the loss discontinuously too. */
    for (uint32_t k = 0; k < count; ++k) sig = (sig ^ order[k]) * 1099511628211ull;
    for (uint32_t i = 0; i < n; ++i) sig = (sig ^ (uint64_t)refs[i].visible) * 1099511628211ull;
    *signature = sig;
  }
  const double values = 3.0 * (double)width * height;
  double result;
  if (lambda <= 0.0) {
    result = weighted_l1 / values;
  } else {
    result = (1.0 - lambda) * weighted_l1 / values +
             lambda * (weight_sum / values - gso_reference_ssim(render, truth, width, height, weights));
  }
  free(render);
  free(truth);
  free(weights);
  free(refs);
  free(order);
  return result;
}
