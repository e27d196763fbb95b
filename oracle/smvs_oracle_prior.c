/*
 * smvs_oracle_prior.c — CPU restatement of the propagate-depth initial maps
 * (PatchMatchACMMCuda::InitWorkspace, src/mvs/patch_match_cuda.cu:603-659).
 *
 * TEST INFRASTRUCTURE ONLY: the checker of sensemap_b200/csrc/smvs_prior.cu,
 * never linked by the product. Compiled with -ffp-contract=off: every float
 * operation below is one IEEE operation in the order the CUDA unit spells it,
 * so the GPU maps are compared bit for bit.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "orc_pose.h"
#include "smvs_oracle.h"

static inline float texel(const float* d, int w, int h, int x, int y) {
  return (x >= 0 && x < w && y >= 0 && y < h) ? d[(size_t)y * w + x] : 0.0f;
}

/* GenerateProjectDepthMaps, kernel_functions.cu:778-826, for one source. */
static void project_depth(const float* sdepth, int sw, int sh, int grid_w, int grid_h, const float* pose, int W,
                          int H, const float refK[4], float* comp) {
  const float* iP = pose + 31; /* P^-1 */
  for (int row = 0; row < grid_h; ++row)
    for (int col = 0; col < grid_w; ++col) {
      /* The linear texture read at the integer coordinate: the four texels
       * around the pixel corner with weights 1/4 (border 0), summed in double
       * and rounded once. */
      const double sum = (double)texel(sdepth, sw, sh, col - 1, row - 1) + (double)texel(sdepth, sw, sh, col, row - 1) +
                         (double)texel(sdepth, sw, sh, col - 1, row) + (double)texel(sdepth, sw, sh, col, row);
      const float depth = (float)(sum * 0.25);
      if (depth < 1e-6f) continue;
      /* [quirk] kernel_functions.cu:803-804 stores the products back into the int
       * pixel indices (col *= depth), truncating them toward zero. */
      const float c = (float)(int)((float)col * depth), r = (float)(int)((float)row * depth);
      const float bx = iP[0] * c + iP[1] * r + iP[2] * depth + iP[3];
      const float by = iP[4] * c + iP[5] * r + iP[6] * depth + iP[7];
      const float bz = iP[8] * c + iP[9] * r + iP[10] * depth + iP[11];
      const float ibz = 1.0f / bz;
      const float bcol = ibz * refK[0] * bx + refK[1];
      const float brow = ibz * refK[2] * by + refK[3];
      if (!(bcol >= 0.0f && bcol < (float)W && brow >= 0.0f && brow < (float)H)) continue;
      const size_t q = (size_t)(int)brow * W + (size_t)(int)bcol;
      /* atomicMin on the bits: the smaller bit pattern (positive floats order). */
      uint32_t a, b;
      memcpy(&a, &comp[q], 4);
      memcpy(&b, &bz, 4);
      if (b < a) comp[q] = bz;
    }
}

/* EstimatePatchNormal, kernel_functions.cu:864-909. */
static int patch_normal(const float* depth, int W, int H, int row, int col, const float iK[4], float n[3]) {
  if (col >= W - 1 || row >= H - 1 || col <= 0 || row <= 0) return 0;
  const float d = depth[(size_t)row * W + col];
  if (d <= 0) return 0;
  const int nr[4] = {row - 1, row, row + 1, row};
  const int nc[4] = {col, col + 1, col, col - 1};
  float p[4][3];
  for (int k = 0; k < 4; ++k) {
    const float nd = depth[(size_t)nr[k] * W + nc[k]];
    if ((double)(fabsf(nd - d) / d) > 0.02) return 0;
    p[k][0] = nd * (iK[0] * (float)nc[k] + iK[1]); /* ComputePointAtDepth :308-315 */
    p[k][1] = nd * (iK[2] * (float)nr[k] + iK[3]);
    p[k][2] = nd;
  }
  const float u[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
  const float v[3] = {p[1][0] - p[3][0], p[1][1] - p[3][1], p[1][2] - p[3][2]};
  n[0] = u[1] * v[2] - u[2] * v[1];
  n[1] = u[2] * v[0] - u[0] * v[2];
  n[2] = u[0] * v[1] - u[1] * v[0];
  const float inv = 1.0f / sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] *= inv; n[1] *= inv; n[2] *= inv;
  return 1;
}

static void bubble(float* a, int n) { /* BubbleSort, utils.h */
  for (int i = 0; i < n - 1; ++i)
    for (int j = 0; j < n - 1 - i; ++j)
      if (a[j] > a[j + 1]) { const float t = a[j]; a[j] = a[j + 1]; a[j + 1] = t; }
}

int orc_propagate_init(int W, int H, int N, const float refK[4], const float refiK[4], const float* poses,
                       const smvs_view* src, float* depth, float* normal, float* prior) {
  if (W <= 0 || H <= 0 || N < 1 || N > SMVS_MAX_SRC || !poses || !src || !depth || !normal || !prior)
    return SMVS_EINVAL;
  const size_t WH = (size_t)W * H;
  int gw = 0, gh = 0; /* the sources' common grid, patch_match_cuda.cu:606-620 */
  for (int i = 0; i < N; ++i) {
    if (src[i].width > gw) gw = src[i].width;
    if (src[i].height > gh) gh = src[i].height;
  }
  float* comp = (float*)malloc(sizeof(float) * (size_t)N * WH);
  if (!comp) return SMVS_ENOMEM;
  for (size_t i = 0; i < (size_t)N * WH; ++i) comp[i] = FLT_MAX;
  for (int i = 0; i < N; ++i)
    if (src[i].depth)
      project_depth(src[i].depth, src[i].width, src[i].height, gw, gh, poses + (size_t)i * SMVS_POSE_FLOATS, W, H,
                    refK, comp + (size_t)i * WH);
  /* CompositeInitDepthMap, kernel_functions.cu:827-862. */
  memset(prior, 0, sizeof(float) * WH);
  for (size_t pix = 0; pix < WH; ++pix) {
    if (depth[pix] > 0) continue;
    float d[SMVS_MAX_SRC];
    int n = 0;
    for (int i = 0; i < N; ++i) {
      const float v = comp[(size_t)i * WH + pix];
      if (v > 0 && v < FLT_MAX) d[n++] = v;
    }
    if (n > 2) {
      bubble(d, n);
      const float m = d[n / 2];
      depth[pix] = m;
      int consistent = 0;
      for (int i = 0; i < n; ++i) consistent += ((double)(fabsf(d[i] - m) / m) <= 0.01) ? 1 : 0;
      if (consistent > 2) prior[pix] = m;
    } else if (n > 0) {
      depth[pix] = (n > 1) ? fminf(d[0], d[1]) : d[0];
    }
  }
  free(comp);
  /* CompositeInitNormalMap, kernel_functions.cu:911-966: every pixel reads
   * only the depth map, so the order of pixels does not matter. */
  const int dr[5] = {0, -1, -1, 1, 1}, dc[5] = {0, -1, 1, 1, -1};
  for (int row = 0; row < H; ++row)
    for (int col = 0; col < W; ++col) {
      float c[3][5];
      int n = 0;
      for (int k = 0; k < 5; ++k) {
        float e[3];
        if (patch_normal(depth, W, H, row + dr[k], col + dc[k], refiK, e)) {
          c[0][n] = e[0]; c[1][n] = e[1]; c[2][n] = e[2];
          n++;
        }
      }
      if (n == 0) continue;
      for (int a = 0; a < 3; ++a) bubble(c[a], n);
      const int m = n >> 1;
      const float v[3] = {c[0][m], c[1][m], c[2][m]};
      const float inv = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      const size_t pix = (size_t)row * W + col;
      normal[pix] = v[0] * inv;
      normal[WH + pix] = v[1] * inv;
      normal[2 * WH + pix] = v[2] * inv;
    }
  return SMVS_OK;
}

int orc_propagate_init_problem(const smvs_problem* p, float* depth, float* normal, float* prior) {
  if (!p || p->memory != SMVS_MEM_HOST || !p->ref.depth || !p->ref.normal) return SMVS_EINVAL;
  if (p->num_src < 1 || p->num_src > SMVS_MAX_SRC) return SMVS_EINVAL;
  const size_t WH = (size_t)p->ref.width * p->ref.height;
  float refK[4], refiK[4];
  float* poses = (float*)malloc(sizeof(float) * SMVS_POSE_FLOATS * p->num_src);
  if (!poses) return SMVS_ENOMEM;
  build_poses(p, refK, refiK, poses);
  memcpy(depth, p->ref.depth, sizeof(float) * WH);
  memcpy(normal, p->ref.normal, sizeof(float) * 3 * WH);
  const int st = orc_propagate_init(p->ref.width, p->ref.height, p->num_src, refK, refiK, poses, p->src, depth,
                                    normal, prior);
  free(poses);
  return st;
}
