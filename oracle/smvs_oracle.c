/*
 * smvs_oracle.c — OpenMP transcription of the reference kernel logic.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the timed CPU
 * baseline; never part of the product path. Every function cites the
 * reference file:line it restates (paths relative to the SenseMap tree).
 * Quirks of the reference are kept on purpose and marked "[quirk]".
 */
#include "smvs_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_HYP 11 /* K_NUM_SAMPS + 3, kernel_functions.h:32 */
#define ORC_MAX_WIN 15 /* 2*7+1, largest supported window */
#define ORC_MARSAGLIA_TRIALS 32

/* ------------------------------------------------------------------------ */
/* Counter-based RNG (replaces cuRAND, gpu_mat_prng.cu:10-37).               */
/* ------------------------------------------------------------------------ */
static inline uint64_t mix64(uint64_t z) { /* splitmix64 finaliser */
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static inline uint64_t stage_key(uint64_t seed, uint32_t stage) {
  return mix64(seed + 0x632BE59BD9B4E019ULL * (uint64_t)(stage + 1u));
}
typedef struct { uint64_t key; uint32_t draw; } rng_t;
static inline rng_t rng_make(uint64_t skey, uint32_t pixel) {
  rng_t r; r.key = mix64(skey + (uint64_t)pixel); r.draw = 0; return r;
}
static inline float rng_uniform(rng_t* r) { /* (0, 1], like curand_uniform */
  uint64_t x = mix64(r->key + 0x9E3779B97F4A7C15ULL * (uint64_t)(r->draw + 1u));
  r->draw++;
  return (float)((x >> 40) + 1u) * (1.0f / 16777216.0f);
}
float orc_uniform(uint64_t seed, uint32_t stage, uint32_t pixel, uint32_t draw) {
  rng_t r = rng_make(stage_key(seed, stage), pixel); r.draw = draw; return rng_uniform(&r);
}
/* Stage numbering shared with the engine. */
#define STAGE_INIT 1u
static inline uint32_t stage_sweep(int iter, int colour) { return 2u + 4u * (uint32_t)iter + (uint32_t)colour; }
static inline uint32_t stage_local(int iter, int colour) { return 4u + 4u * (uint32_t)iter + (uint32_t)colour; }

/* ------------------------------------------------------------------------ */
/* Small helpers                                                              */
/* ------------------------------------------------------------------------ */
static inline int f2i_rz(float x) { /* cvt.rzi.s32.f32: saturating, NaN -> 0 */
  if (x != x) return 0;
  if (x >= 2147483647.0f) return INT_MAX;
  if (x <= -2147483648.0f) return INT_MIN;
  return (int)x;
}
static inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Round a float to the nearest FP16 value (round-to-nearest-even), for the
 * precision form's FP16 storage. Inputs are in [0, 1] (no overflow). */
static float round_to_half(float f) {
  union { float f; uint32_t u; } v = {f};
  const uint32_t sign = v.u & 0x80000000u;
  uint32_t a = v.u & 0x7fffffffu;
  const int exp = (int)(a >> 23) - 127;
  if (a == 0 || exp >= 16) return f;
  if (exp < -14) {  /* subnormal half: quantum 2^-24 */
    const float q = nearbyintf(fabsf(f) * 16777216.0f) / 16777216.0f;
    return sign ? -q : q;
  }
  /* keep 10 mantissa bits, round to nearest even */
  const uint32_t lsb = (a >> 13) & 1u;
  a += 0x0fffu + lsb;
  a &= ~0x1fffu;
  v.u = sign | a;
  return v.f;
}

/* CUDA texture linear filtering, unnormalised coordinates, border address mode
 * (zero outside), as configured at patch_match_cuda.cu:258-278 and :355-360.
 * The fractional positions are rounded to 8 bits (A, B in 0..256, CUDA C
 * Programming Guide, "Texture Fetching"); measured on B200 (sm_100a), the four
 * weights are then integers in 1/256 units with w11 = round(A*B/256) and the
 * others by subtraction (so ties resolve the way the hardware does), and the
 * weighted sum is exact for FP32 texels. FP16 texels return an FP16-rounded
 * result (half_out). */
static float tex_bilinear_mode(const float* img, int w, int h, float x, float y, int half_out) {
  if (!(x > -1.0e7f && x < 1.0e7f && y > -1.0e7f && y < 1.0e7f)) return 0.0f;
  const float xb = x - 0.5f, yb = y - 0.5f;
  const float fx = floorf(xb), fy = floorf(yb);
  const int i = (int)fx, j = (int)fy;
  const int A = (int)floorf((xb - fx) * 256.0f + 0.5f);
  const int B = (int)floorf((yb - fy) * 256.0f + 0.5f);
  const int w11 = (A * B + 128) >> 8, w10 = A - w11, w01 = B - w11, w00 = 256 - A - B + w11;
  float t00 = 0, t10 = 0, t01 = 0, t11 = 0;
  const int in_i0 = (i >= 0 && i < w), in_i1 = (i + 1 >= 0 && i + 1 < w);
  if (j >= 0 && j < h) {
    if (in_i0) t00 = img[(size_t)j * w + i];
    if (in_i1) t10 = img[(size_t)j * w + i + 1];
  }
  if (j + 1 >= 0 && j + 1 < h) {
    if (in_i0) t01 = img[(size_t)(j + 1) * w + i];
    if (in_i1) t11 = img[(size_t)(j + 1) * w + i + 1];
  }
  const double v = ((double)w00 * t00 + (double)w10 * t10 + (double)w01 * t01 + (double)w11 * t11) / 256.0;
  return half_out ? round_to_half((float)v) : (float)v;
}

float orc_tex_bilinear(const float* img, int w, int h, float x, float y) {
  return tex_bilinear_mode(img, w, h, x, y, 0);
}

/* Exact bilinear in double (FP64 evaluator). */
static double tex_bilinear_f64(const float* img, int w, int h, double x, double y) {
  if (!(x > -1.0e7 && x < 1.0e7 && y > -1.0e7 && y < 1.0e7)) return 0.0;
  const double xb = x - 0.5, yb = y - 0.5;
  const double fx = floor(xb), fy = floor(yb);
  const int i = (int)fx, j = (int)fy;
  const double a = xb - fx, b = yb - fy;
  double t[4] = {0, 0, 0, 0};
  for (int dj = 0; dj < 2; ++dj)
    for (int di = 0; di < 2; ++di) {
      int ii = i + di, jj = j + dj;
      if (ii >= 0 && ii < w && jj >= 0 && jj < h) t[dj * 2 + di] = img[(size_t)jj * w + ii];
    }
  return (1 - a) * (1 - b) * t[0] + a * (1 - b) * t[1] + (1 - a) * b * t[2] + a * b * t[3];
}

/* ------------------------------------------------------------------------ */
/* Context                                                                    */
/* ------------------------------------------------------------------------ */
typedef struct {
  int W, H, N, R, S;
  /* SweepOptions (kernel_functions.h:67-111) as filled at patch_match_cuda.cu:914-950 */
  float sn, cn;                  /* BilateralWeightComputer normalisations (utils.h:72-92) */
  double sigma_s, sigma_c;       /* the options' sigmas, for the FP64 evaluator */
  float depth_min, depth_max;
  int num_samples, thk, num_good, num_bad, random_opt, local_opt, geom, num_iter;
  float geom_reg, geom_max, rand_depth_ratio, rand_a1, rand_a2, init_mc, max_mc, alpha, beta;
  uint64_t seed;
  float refK[4], refiK[4];
  float* poses;                  /* N*43 */
  float* ref;                    /* W*H, [0,1] */
  float* ref_sum;                /* W*H */
  float* ref_sqsum;              /* W*H */
  float* grad;                   /* W*H */
  float* src[SMVS_MAX_SRC];
  int sw[SMVS_MAX_SRC], sh[SMVS_MAX_SRC];
  int src_half;                  /* FP16 source storage: filtered values are FP16 */
  float* sdepth[SMVS_MAX_SRC];   /* geometric pass only */
  /* Prior maps (SweepOptions::prior_depth_ncc / propagate_depth): mode 1 =
   * has_prior_depth, 2 = propagate_depth; NULL normal/weight maps read as 0. */
  int prior_mode;
  const float* prior_depth;
  const float* prior_normal;
  const float* prior_wgt;
  /* state */
  float *depth, *normal, *conf, *cost;
  uint32_t* view_sel;
} ctx_t;

static const float kMWeights[5] = {0.f, 1.f, 2.01f, 3.03f, 4.06f}; /* kernel_functions.cu:22 */
static const int kNeighborOffs[8][2] = {{0, -1}, {-1, 0}, {0, 1}, {1, 0},
                                        {-1, -1}, {-1, 1}, {1, 1}, {1, -1}}; /* :23-25 */
static const int kDirSamples[8][20] = {                                      /* :27-44 */
    {-1, -2, 1, -2, -2, -3, 2, -3, -3, -4, 3, -4, -4, -5, 4, -5, -5, -6, 5, -6},
    {-1, 2, 1, 2, -2, 3, 2, 3, -3, 4, 3, 4, -4, 5, 4, 5, -5, 6, 5, 6},
    {-2, -1, -2, 1, -3, -2, -3, 2, -4, -3, -4, 3, -5, -4, -5, 4, -6, -5, -6, 5},
    {2, -1, 2, 1, 3, -2, 3, 2, 4, -3, 4, 3, 5, -4, 5, 4, 6, -5, 6, 5},
    {0, -3, 0, -5, 0, -7, 0, -9, 0, -11, 0, -13, 0, -15, 0, -17, 0, -19, 0, -21},
    {0, 3, 0, 5, 0, 7, 0, 9, 0, 11, 0, 13, 0, 15, 0, 17, 0, 19, 0, 21},
    {-3, 0, -5, 0, -7, 0, -9, 0, -11, 0, -13, 0, -15, 0, -17, 0, -19, 0, -21, 0},
    {3, 0, 5, 0, 7, 0, 9, 0, 11, 0, 13, 0, 15, 0, 17, 0, 19, 0, 21, 0}};
static const float kScharrX[3][3] = {{-3, 0, 3}, {-10, 0, 10}, {-3, 0, 3}}; /* :56-60 */
static const float kScharrY[3][3] = {{-3, -10, -3}, {0, 0, 0}, {3, 10, 3}};
#define DEG2RAD_D(deg) ((deg) * 0.0174532925199432) /* kernel_functions.h:39 */

static inline float ref_at(const ctx_t* c, int r, int col) { /* point sample, border 0 */
  if (r < 0 || r >= c->H || col < 0 || col >= c->W) return 0.0f;
  return c->ref[(size_t)r * c->W + col];
}

#include "orc_pose.h"

/* ------------------------------------------------------------------------ */
/* Device helpers restated                                                    */
/* ------------------------------------------------------------------------ */
/* ComposeHomography, kernel_functions.cu:431-503 (same expression order). */
static void compose_homography(const float* pose, int row, int col, float depth, const float n[3],
                               const float* iK, float H[9]) {
  const float* K = pose;
  const float* R = pose + 4;
  const float* T = pose + 13;
  const float dist = depth * (n[0] * (iK[0] * col + iK[1]) + n[1] * (iK[2] * row + iK[3]) + n[2]);
  const float inv_dist = 1.0f / dist;
  const float N0 = inv_dist * n[0], N1 = inv_dist * n[1], N2 = inv_dist * n[2];
  const float N0T0 = N0 * T[0], N0T1 = N0 * T[1], N0T2 = N0 * T[2];
  const float N1T0 = N1 * T[0], N1T1 = N1 * T[1], N1T2 = N1 * T[2];
  const float N2T0 = N2 * T[0], N2T1 = N2 * T[1], N2T2 = N2 * T[2];
  const float K0R0N0T0 = K[0] * (R[0] + N0T0);
  const float K0R1N1T0 = K[0] * (R[1] + N1T0);
  const float K2R3N0T1 = K[2] * (R[3] + N0T1);
  const float K2R4N1T1 = K[2] * (R[4] + N1T1);
  const float K1R6N0T2 = K[1] * (R[6] + N0T2);
  const float K1R7N1T2 = K[1] * (R[7] + N1T2);
  const float K3R6N0T2 = K[3] * (R[6] + N0T2);
  const float K3R7N1T2 = K[3] * (R[7] + N1T2);
  const float A = K0R0N0T0 + K1R6N0T2;
  const float B = K0R1N1T0 + K1R7N1T2;
  const float C = K2R3N0T1 + K3R6N0T2;
  const float D = K2R4N1T1 + K3R7N1T2;
  const float R8 = R[8] + N2T2;
  H[0] = iK[0] * A;
  H[1] = iK[2] * B;
  H[2] = K[0] * (R[2] + N2T0) + K[1] * R8 + iK[1] * A + iK[3] * B;
  H[3] = iK[0] * C;
  H[4] = iK[2] * D;
  H[5] = K[2] * (R[5] + N2T1) + K[3] * R8 + iK[1] * C + iK[3] * D;
  H[6] = iK[0] * (R[6] + N0T2);
  H[7] = iK[2] * (R[7] + N1T2);
  H[8] = iK[1] * (R[6] + N0T2) + iK[3] * (R[7] + N1T2) + R8;
}

/* Per-pixel reference data used by every cost evaluation. */
typedef struct {
  float center, rsum, rsq, rvar;
  float win[ORC_MAX_WIN * ORC_MAX_WIN]; /* ref window, border 0 */
} pixref_t;

static void load_pixref(const ctx_t* c, int row, int col, pixref_t* pr) {
  const size_t pix = (size_t)row * c->W + col;
  pr->center = c->ref[pix];
  pr->rsum = c->ref_sum[pix];
  pr->rsq = c->ref_sqsum[pix];
  pr->rvar = pr->rsq - pr->rsum * pr->rsum;
  const int R = c->R, D = 2 * R + 1;
  for (int dr = -R; dr <= R; ++dr)
    for (int dc = -R; dc <= R; ++dc) pr->win[(dr + R) * D + (dc + R)] = ref_at(c, row + dr, col + dc);
}

/* ComputeNCCCost<R,S>, kernel_functions.cu:1245-1340 (incremental homography). */
static float ncc_cost(const ctx_t* c, int v, int row, int col, float depth, const float n[3],
                      const pixref_t* pr) {
  const float kMaxCost = 2.0f;
  const int R = c->R, S = c->S, D = 2 * R + 1;
  float H[9];
  compose_homography(c->poses + (size_t)v * SMVS_POSE_FLOATS, row, col, depth, n, c->refiK, H);
  const float inv_z0 = 1.0f / (H[6] * col + H[7] * row + H[8]);
  const int u = f2i_rz((H[0] * col + H[1] * row + H[2]) * inv_z0);
  const int vv = f2i_rz((H[3] * col + H[4] * row + H[5]) * inv_z0);
  /* [quirk] bounds are the reference image's width/height (:1265-1270) */
  if (u < 0 || u >= c->W || vv < 0 || vv >= c->H) return kMaxCost;
  const int row_start = row - R, col_start = col - R;
  float col_src = H[0] * col_start + H[1] * row_start + H[2];
  float row_src = H[3] * col_start + H[4] * row_start + H[5];
  float z = H[6] * col_start + H[7] * row_start + H[8];
  float bcol = col_src, brow = row_src, bz = z;
  float Hs[9];
  for (int k = 0; k < 9; ++k) Hs[k] = (float)S * H[k];
  float ss = 0, sss = 0, srs = 0, sw = 0;
  const float* img = c->src[v];
  const int w = c->sw[v], h = c->sh[v];
  for (int dr = -R; dr <= R; dr += S) {
    for (int dc = -R; dc <= R; dc += S) {
      const float iz = 1.0f / z;
      const float fu = iz * col_src + 0.5f;
      const float fv = iz * row_src + 0.5f;
      const float rc = pr->win[(dr + R) * D + (dc + R)];
      const float sc = tex_bilinear_mode(img, w, h, fu, fv, c->src_half);
      const float cd = pr->center - rc;
      const float wgt = expf(-(float)(dr * dr + dc * dc) * c->sn - cd * cd * c->cn);
      const float wsc = wgt * sc;
      ss += wsc;
      sss += wsc * sc;
      srs += wsc * rc;
      sw += wgt;
      col_src += Hs[0];
      row_src += Hs[3];
      z += Hs[6];
    }
    bcol += Hs[1]; brow += Hs[4]; bz += Hs[7];
    col_src = bcol; row_src = brow; z = bz;
  }
  const float isw = 1.0f / sw;
  ss *= isw; sss *= isw; srs *= isw;
  const float svar = sss - ss * ss;
  if (pr->rvar < 1e-5f || svar < 1e-5f) return kMaxCost;
  const float cov = srs - pr->rsum * ss;
  const float val = 1.0f - cov * (1.0f / sqrtf(pr->rvar * svar));
  return fmaxf(0.0f, fminf(kMaxCost, val));
}

/* ComputeGeomConsistencyCostShared, kernel_functions.cu:505-568. K = {fx,cx,fy,cy}
 * of the reference (the sweep passes &ref_invK[4]); see local_opt for the quirk. */
static float geom_cost(const ctx_t* c, int v, float row, float col, float depth, const float np[3],
                       const float K[4]) {
  const float* pose = c->poses + (size_t)v * SMVS_POSE_FLOATS;
  const float* P = pose + 19;
  const float* iP = pose + 31;
  const float X0 = depth * np[0], X1 = depth * np[1], X2 = depth * np[2];
  const float ifz = 1.0f / (P[8] * X0 + P[9] * X1 + P[10] * X2 + P[11]);
  float scol = ifz * (P[0] * X0 + P[1] * X1 + P[2] * X2 + P[3]);
  float srow = ifz * (P[4] * X0 + P[5] * X1 + P[6] * X2 + P[7]);
  const float sd = orc_tex_bilinear(c->sdepth[v], c->sw[v], c->sh[v], scol + 0.5f, srow + 0.5f);
  if (sd == 0.0f) return c->geom_max;
  scol *= sd; srow *= sd;
  const float bx = iP[0] * scol + iP[1] * srow + iP[2] * sd + iP[3];
  const float by = iP[4] * scol + iP[5] * srow + iP[6] * sd + iP[7];
  const float bz = iP[8] * scol + iP[9] * srow + iP[10] * sd + iP[11];
  const float ibz = 1.0f / bz;
  const float bcol = ibz * K[0] * bx + K[1];
  const float brow = ibz * K[2] * by + K[3];
  const float dc = col - bcol, dr = row - brow;
  return fminf(c->geom_max, sqrtf(dc * dc + dr * dr));
}

/* A pixel's prior: normal xyz, depth w and weight (kernel_functions.cu:
 * 1533-1543, 2188-2200). */
typedef struct { float x, y, z, w, wgt; } prior_t;

static prior_t load_prior(const ctx_t* c, size_t pix) {
  prior_t pi = {0, 0, 0, 0, 0};
  if (c->prior_mode == 0) return pi;
  const size_t WH = (size_t)c->W * c->H;
  pi.w = c->prior_depth[pix];
  if (c->prior_normal) {
    pi.x = c->prior_normal[pix]; pi.y = c->prior_normal[WH + pix]; pi.z = c->prior_normal[2 * WH + pix];
  }
  if (c->prior_wgt) pi.wgt = c->prior_wgt[pix];
  return pi;
}

/* ComputeNCCWeightFromPrior (kernel_functions.cu:316-340) times the
 * PRIOR_WGT_COST factor (:1470-1478), with the reference's float/double mix;
 * 1 unless mode 1 and a prior depth above FLT_EPSILON. */
static float prior_weight(const ctx_t* c, const prior_t* pi, const float h[3], float hd, float rvar) {
  if (c->prior_mode != 1 || !(pi->w > FLT_EPSILON)) return 1.0f;
  float regu = 1.0f;
  const float sigma2 = (float)(0.5 - 0.4 * exp(-10000.0 * (double)fabsf(rvar)));
  const float dd = hd - pi->w;
  const float dd2 = fmaxf(dd * dd, 0.05f * 0.05f);
  regu = (float)((double)regu * fmax(1.0 - 0.2 * (double)expf(-dd2 / sigma2), 0.01));
  const float pn = pi->x * pi->x + pi->y * pi->y + pi->z * pi->z;
  if ((double)pn > 0.8 && (double)pn < 1.25) {
    const float ct = pi->x * h[0] + pi->y * h[1] + pi->z * h[2];
    const float dt2 = (1.0f - ct) * (1.0f - ct);
    regu = (float)((double)regu * fmax(1.0 - 0.54 * (double)expf(-dt2 / sigma2), 0.01));
  }
  if ((double)pi->wgt < 1.0 && (double)pi->wgt > 0.0) regu = (float)((double)regu * (1.0 - (double)pi->wgt * 0.3));
  return regu;
}

/* ComputeMultiViewCostVector, kernel_functions.cu:1447-1495; pw = the prior
 * factor of the hypothesis (1 without a prior). */
static void cost_vector(const ctx_t* c, int row, int col, float depth, const float n[3],
                        const float np[3], const pixref_t* pr, float* out, float pw) {
  for (int v = 0; v < c->N; ++v) {
    float cost = ncc_cost(c, v, row, col, depth, n, pr) * pw;
    if (c->geom) cost += c->geom_reg * geom_cost(c, v, (float)row, (float)col, depth, np, c->refK);
    out[v] = cost;
  }
}

/* GenerateRandomNormal (view-ray form), kernel_functions.cu:112-139. */
static void random_normal(rng_t* r, const float view_ray[3], float n[3]) {
  float v1 = 0, v2 = 0, s = 2.0f;
  for (int t = 0; t < ORC_MARSAGLIA_TRIALS && s >= 1.0f; ++t) {
    v1 = 2.0f * rng_uniform(r) - 1.0f;
    v2 = 2.0f * rng_uniform(r) - 1.0f;
    s = v1 * v1 + v2 * v2;
  }
  if (s >= 1.0f) { n[0] = 0; n[1] = 0; n[2] = -1.0f; return; }
  const float s_norm = 2.0f * sqrtf(1.0f - s);
  n[0] = v1 * s_norm; n[1] = v2 * s_norm; n[2] = 1.0f - 2.0f * s;
  if (dot3(n, view_ray) > 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
}

/* CorrectNormal, kernel_functions.cu:227-306. */
static void correct_normal(float n[3], const float vd[3], float inv_view_len) {
  const float cal = dot3(n, vd);
  if (cal >= 0) {
    float c3[3];
    c3[0] = n[1] * vd[2] - n[2] * vd[1];
    c3[1] = n[2] * vd[0] - n[0] * vd[2];
    c3[2] = n[0] * vd[1] - n[1] * vd[0];
    float phi = (float)((double)acosf(cal * inv_view_len) - DEG2RAD_D(90.f));
    phi = fminf(phi * 1.01f, -0.001f);
    if (phi == 0) return;
    const float icl = 1.0f / sqrtf(c3[0] * c3[0] + c3[1] * c3[1] + c3[2] * c3[2]);
    c3[0] *= icl; c3[1] *= icl; c3[2] *= icl;
    float om[9] = {0.0f, -c3[2], c3[1], c3[2], 0.0f, -c3[0], -c3[1], c3[0], 0.0f};
    const float sp = sinf(phi);
    float sO[9];
    for (int k = 0; k < 9; ++k) sO[k] = om[k] * sp;
    const float cp = 1.0f - cosf(phi);
    float cO[9];
    cO[0] = cp * (om[0] * om[0] + om[1] * om[3] + om[2] * om[6]);
    cO[1] = cp * (om[0] * om[1] + om[1] * om[4] + om[2] * om[7]);
    cO[2] = cp * (om[0] * om[2] + om[1] * om[5] + om[2] * om[8]);
    cO[3] = cp * (om[3] * om[0] + om[4] * om[3] + om[5] * om[6]);
    cO[4] = cO[3]; /* [quirk] :272-276 copy entries instead of computing them */
    cO[5] = cO[3];
    cO[6] = cp * (om[6] * om[0] + om[7] * om[3] + om[8] * om[6]);
    cO[7] = cO[6];
    cO[8] = cO[6];
    float Rt[9];
    Rt[0] = 1 + sO[0] + cO[0]; Rt[1] = 0 + sO[1] + cO[1]; Rt[2] = 0 + sO[2] + cO[2];
    Rt[3] = 0 + sO[3] + cO[3]; Rt[4] = 1 + sO[4] + cO[4]; Rt[5] = 0 + sO[5] + cO[5];
    Rt[6] = 0 + sO[6] + cO[6]; Rt[7] = 0 + sO[7] + cO[7]; Rt[8] = 1 + sO[8] + cO[8];
    const float r0 = Rt[0] * n[0] + Rt[1] * n[1] + Rt[2] * n[2];
    const float r1 = Rt[3] * n[0] + Rt[4] * n[1] + Rt[5] * n[2];
    const float r2 = Rt[6] * n[0] + Rt[7] * n[1] + Rt[8] * n[2];
    n[0] = r0; n[1] = r1; n[2] = r2;
  }
}

/* PropagateDepth (normalised-point form), kernel_functions.cu:409-429. */
static float propagate_depth(float d1, const float n1[3], const float iK[4], int row1, int col1,
                             const float p2[3]) {
  const float x1 = d1 * (iK[0] * col1 + iK[1]);
  const float y1 = d1 * (iK[2] * row1 + iK[3]);
  const float z1 = d1;
  const float d = n1[0] * x1 + n1[1] * y1 + n1[2] * z1;
  const float t = d / (n1[0] * p2[0] + n1[1] * p2[1] + n1[2] * p2[2]);
  if (fabsf(t) < 1e-5f) return d1;
  return t;
}

/* Normal2Dir / Dir2Normal, utils.h:94-106; PerturbNormal (ACMH form),
 * kernel_functions.cu:214-225. */
static void perturb_normal_acmh(const float n[3], float out[3], float a1, float a2, rng_t* r) {
  const float y = atan2f(sqrtf(n[0] * n[0] + n[1] * n[1]), n[2]);
  const float x = atan2f(n[1], n[0]);
  const float nx = a1 * (2 * rng_uniform(r) - 1) + x;
  const float ny = a2 * (2 * rng_uniform(r) - 1) + y;
  const float sy = sinf(ny);
  out[0] = cosf(nx) * sy;
  out[1] = sinf(nx) * sy;
  out[2] = cosf(ny);
}

static inline int find_min_cost(const float* costs, int n) { /* FindMinCost :648-659 ('<=') */
  float m = FLT_MAX;
  int idx = -1;
  for (int i = 0; i < n; ++i)
    if (costs[i] <= m) { m = costs[i]; idx = i; }
  return idx;
}

/* ------------------------------------------------------------------------ */
/* Kernels restated                                                           */
/* ------------------------------------------------------------------------ */
/* GpuMatRefImage::FilterKernel, gpu_mat_ref_image.cu:16-56 and ComputeGradientMap,
 * kernel_functions.cu:1655-1675. */
static void prep_ref(ctx_t* c) {
  const int W = c->W, H = c->H, R = c->R, S = c->S;
#pragma omp parallel for schedule(static)
  for (int row = 0; row < H; ++row)
    for (int col = 0; col < W; ++col) {
      const float center = ref_at(c, row, col);
      float cs = 0, css = 0, ws = 0;
      for (int wr = -R; wr <= R; wr += S)
        for (int wc = -R; wc <= R; wc += S) {
          const float color = ref_at(c, row + wr, col + wc);
          const float cd = center - color;
          const float w = expf(-(float)(wr * wr + wc * wc) * c->sn - cd * cd * c->cn);
          cs += w * color;
          css += w * color * color;
          ws += w;
        }
      cs /= ws;
      css /= ws;
      c->ref_sum[(size_t)row * W + col] = cs;
      c->ref_sqsum[(size_t)row * W + col] = css;
      float gx = 0, gy = 0;
      for (int dr = -1; dr <= 1; ++dr)
        for (int dc = -1; dc <= 1; ++dc) {
          const float color = ref_at(c, row + dr, col + dc);
          gx += color * kScharrX[dr + 1][dc + 1];
          gy += color * kScharrY[dr + 1][dc + 1];
        }
      c->grad[(size_t)row * W + col] = sqrtf(gx * gx + gy * gy);
    }
}


/* InitWorkspace, patch_match_cuda.cu:582-698: random branch = FillWithRandomNumbers
 * (util/gpu_mat.h:114-130) + InitNormalMap (kernel_functions.cu:689-701); given-map
 * branch = InitDepthMap (kernel_functions.cu:703-737). */
static void init_workspace(ctx_t* c, int random_init, const float* init_depth, const float* init_normal,
                           float opt_dmin, float opt_dmax) {
  const int W = c->W, H = c->H;
  const size_t WH = (size_t)W * H;
  const uint64_t sk = stage_key(c->seed, STAGE_INIT);
#pragma omp parallel for schedule(static)
  for (int row = 0; row < H; ++row)
    for (int col = 0; col < W; ++col) {
      const size_t pix = (size_t)row * W + col;
      rng_t r = rng_make(sk, (uint32_t)pix);
      const float vd[3] = {c->refiK[0] * col + c->refiK[1], c->refiK[2] * row + c->refiK[3], 1.0f};
      float d, n[3];
      if (random_init) {
        d = rng_uniform(&r) * (opt_dmax - opt_dmin) + opt_dmin;
        random_normal(&r, vd, n);
      } else {
        d = init_depth[pix];
        n[0] = init_normal[pix]; n[1] = init_normal[WH + pix]; n[2] = init_normal[2 * WH + pix];
        if (d <= 0) {
          d = rng_uniform(&r) * (opt_dmax - opt_dmin) + opt_dmin;
          random_normal(&r, vd, n);
        }
        if (dot3(n, vd) >= 0) random_normal(&r, vd, n);
      }
      c->depth[pix] = d;
      c->normal[pix] = n[0]; c->normal[WH + pix] = n[1]; c->normal[2 * WH + pix] = n[2];
      c->view_sel[pix] = 0;
    }
}

/* InitConfMapKernel, kernel_functions.cu:1497-1601, over rows
 * [row_begin, row_end). */
static void init_conf(ctx_t* c, int row_begin, int row_end) {
  const int W = c->W, N = c->N;
  const size_t WH = (size_t)W * c->H;
#pragma omp parallel for schedule(dynamic, 4)
  for (int row = row_begin; row < row_end; ++row) {
    pixref_t pr;
    for (int col = 0; col < W; ++col) {
      const size_t pix = (size_t)row * W + col;
      load_pixref(c, row, col, &pr);
      const float np[3] = {c->refiK[0] * col + c->refiK[1], c->refiK[2] * row + c->refiK[3], 1.0f};
      const float n[3] = {c->normal[pix], c->normal[WH + pix], c->normal[2 * WH + pix]};
      float costs[SMVS_MAX_SRC];
      int O[SMVS_MAX_SRC];
      const prior_t pi = load_prior(c, pix);
      cost_vector(c, row, col, c->depth[pix], n, np, &pr, costs,
                  prior_weight(c, &pi, n, c->depth[pix], pr.rvar));
      for (int v = 0; v < N; ++v) { O[v] = v; c->cost[(size_t)v * WH + pix] = costs[v]; }
      /* BubbleSortByValue, utils.h:212-231 */
      for (int i = 0; i < N - 1; ++i)
        for (int j = 0; j < N - 1 - i; ++j)
          if (costs[j] > costs[j + 1]) {
            float t = costs[j]; costs[j] = costs[j + 1]; costs[j + 1] = t;
            int o = O[j]; O[j] = O[j + 1]; O[j + 1] = o;
          }
      float conf = 0.0f;
      uint32_t sel = c->view_sel[pix];
      for (int i = 0; i < c->thk; ++i) { conf += costs[i]; sel |= (1u << O[i]); }
      conf /= kMWeights[c->thk];
      c->conf[pix] = conf;
      c->view_sel[pix] = sel;
    }
  }
}

/* SweepFromCheckerBoardOpt, kernel_functions.cu:2136-2560, for one pixel. */
static void sweep_pixel(ctx_t* c, int row, int col, float th_mc, uint64_t sk) {
  const int W = c->W, H = c->H, N = c->N;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  rng_t r = rng_make(sk, (uint32_t)pix);
  float depth = c->depth[pix];
  float normal[3] = {c->normal[pix], c->normal[WH + pix], c->normal[2 * WH + pix]};
  const float grad = c->grad[pix];
  const prior_t pri = load_prior(c, pix);
  const float prf = (c->prior_mode == 1 && (double)pri.w > 1e-6) ? 0.1f : 1.0f; /* :2201-2203 */
  const float inv_beta2 = 0.5f / (c->beta * c->beta);
  const float depth_min = c->depth_min;
  const float depth_max = (float)(1.2 * (double)c->depth_max); /* [quirk] :2213 */
  const float a1 = fminf(c->rand_a1 * prf, (float)DEG2RAD_D(180.0f));
  const float a2 = fminf(c->rand_a2 * prf, (float)DEG2RAD_D(90.0f));
  const float* iK = c->refiK;
  const float vd[3] = {iK[0] * col + iK[1], iK[2] * row + iK[3], 1.0f};
  const float ivl = 1.0f / sqrtf(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
  const float* np = vd;

  float hyp[ORC_MAX_HYP][4]; /* x y z = normal, w = depth */
  int ns = 0;
  hyp[ns][0] = normal[0]; hyp[ns][1] = normal[1]; hyp[ns][2] = normal[2]; hyp[ns][3] = depth; ns++;

  if (grad >= 1.0f) { /* :2237-2276 */
    float nconf[4], O[4];
    int nvalid = 0;
    for (int i = 0; i < 4; ++i) {
      O[i] = (float)i;
      const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
      if (u < 0 || u >= W || v < 0 || v >= H) { nconf[i] = FLT_MAX; continue; }
      nvalid++;
      nconf[i] = c->conf[(size_t)v * W + u];
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3 - i; ++j)
        if (nconf[j] > nconf[j + 1]) {
          float t = nconf[j]; nconf[j] = nconf[j + 1]; nconf[j + 1] = t;
          t = O[j]; O[j] = O[j + 1]; O[j + 1] = t;
        }
    if (nvalid > 2) nvalid = 2;
    for (int i = 0; i < nvalid; ++i) {
      const int idx = (int)O[i];
      const int u = kNeighborOffs[idx][1] + col, v = kNeighborOffs[idx][0] + row;
      const size_t q = (size_t)v * W + u;
      float nn[3] = {c->normal[q], c->normal[WH + q], c->normal[2 * WH + q]};
      correct_normal(nn, vd, ivl);
      hyp[ns][3] = propagate_depth(c->depth[q], nn, iK, v, u, np);
      hyp[ns][0] = nn[0]; hyp[ns][1] = nn[1]; hyp[ns][2] = nn[2];
      ns++;
    }
  }
  for (int k = 0; k < 8; ++k) { /* :2278-2327 */
    int br = 0, bc = 0;
    float best = FLT_MAX;
    for (int s = 0; s < 10; ++s) {
      const int nr = row + kDirSamples[k][2 * s], nc = col + kDirSamples[k][2 * s + 1];
      if (nr < 0 || nr >= H || nc < 0 || nc >= W) continue;
      float nconf = c->conf[(size_t)nr * W + nc];
      if (c->prior_mode != 0 && c->prior_wgt) { /* PRIOR_WGT_PROGET :2292-2304 */
        const float pws = c->prior_wgt[(size_t)nr * W + nc];
        if ((double)pws > 1e-6) nconf = (float)((double)nconf * (1.0 - 0.2 * (double)pws));
      }
      if (best > nconf) { br = nr; bc = nc; best = nconf; }
    }
    if (best < FLT_MAX) {
      const size_t q = (size_t)br * W + bc;
      float nn[3] = {c->normal[q], c->normal[WH + q], c->normal[2 * WH + q]};
      correct_normal(nn, vd, ivl);
      hyp[ns][3] = propagate_depth(c->depth[q], nn, iK, br, bc, np);
      hyp[ns][0] = nn[0]; hyp[ns][1] = nn[1]; hyp[ns][2] = nn[2];
      ns++;
    }
  }

  pixref_t pr;
  load_pixref(c, row, col, &pr);
  float M[ORC_MAX_HYP][SMVS_MAX_SRC];
  for (int v = 0; v < N; ++v) M[0][v] = c->cost[(size_t)v * WH + pix];
  for (int h = 1; h < ns; ++h)
    cost_vector(c, row, col, hyp[h][3], hyp[h], np, &pr, M[h], prior_weight(c, &pri, hyp[h], hyp[h][3], pr.rvar));

  /* ACMM view selection, :2364-2427 */
  uint32_t flags = 0;
  float probs[SMVS_MAX_SRC];
  for (int v = 0; v < N; ++v) {
    unsigned n1 = 0, n2 = 0;
    probs[v] = 0.0f;
    for (int h = 0; h < ns; ++h) {
      const float cst = M[h][v];
      probs[v] += expf(-cst * cst * inv_beta2);
      n1 += (cst < th_mc);
      n2 += (cst > c->max_mc);
    }
    if ((int)n1 >= c->num_good && (int)n2 <= c->num_bad) flags |= (1u << v);
  }
  for (int v = 0; v < N; ++v)
    if (flags != 0 && !((flags >> v) & 1u)) probs[v] = 0;
  if (flags == 0) return;
  { /* TransformPDFToCDF :673-686 */
    float sum = 0.0f;
    for (int v = 0; v < N; ++v) sum += probs[v];
    const float inv = 1.0f / sum;
    float cum = 0.0f;
    for (int v = 0; v < N; ++v) { cum += probs[v] * inv; probs[v] = cum; }
  }
  float vw[SMVS_MAX_SRC];
  for (int v = 0; v < N; ++v) vw[v] = 0.0f;
  for (int s = 0; s < c->num_samples; ++s) {
    const float rp = rng_uniform(&r) - FLT_EPSILON;
    for (int v = 0; v < N; ++v)
      if (probs[v] > rp) {
        if (c->random_opt) vw[v] = 1.0f; else vw[v] += 1.0f;
        break;
      }
  }
  float wn = 0.0f;
  for (int v = 0; v < N; ++v) wn += vw[v];
  if (wn <= 1e-5f) return;
  const float iwn = 1.0f / wn;
  uint32_t sel = 0;
  for (int v = 0; v < N; ++v) { vw[v] *= iwn; if (vw[v] > 0) sel |= (1u << v); }
  float costs[ORC_MAX_HYP];
  for (int h = 0; h < ns; ++h) {
    float cs = 0;
    for (int v = 0; v < N; ++v) cs += vw[v] * M[h][v];
    costs[h] = cs;
  }
  c->view_sel[pix] = sel;
  int mi = -1;
  if (c->prior_mode == 1 && pri.w > 0.0f) { /* FindMinCostWithin :661-671, band :2431-2437 */
    const float lo = (float)fmin((double)(pri.w * 0.95f) - 0.05, 0.0);
    const float hi = (float)((double)(pri.w * 1.05f) + 0.05);
    float m = FLT_MAX;
    for (int h = 0; h < ns; ++h)
      if (costs[h] <= m && hyp[h][3] >= lo && hyp[h][3] <= hi) { m = costs[h]; mi = h; }
  } else {
    mi = find_min_cost(costs, ns);
  }
  if (mi < 0) return;
  depth = hyp[mi][3];
  normal[0] = hyp[mi][0]; normal[1] = hyp[mi][1]; normal[2] = hyp[mi][2];

  /* Refinement, :2449-2520 */
  float nn[3];
  const float pd_min = (1.0f - c->rand_depth_ratio) * depth, pd_max = (1.0f + c->rand_depth_ratio) * depth;
  const float ndepth = rng_uniform(&r) * (pd_max - pd_min) + pd_min; /* PerturbDepth :141-147 */
  perturb_normal_acmh(normal, nn, a1, a2, &r);
  correct_normal(nn, vd, ivl);
  const int rand_depth = !(c->prior_mode == 2 && pri.w > 0.0f); /* :2467-2486 */
  const float rdepth = rand_depth ? rng_uniform(&r) * (depth_max - depth_min) + depth_min : 0.0f;
  float rn[3];
  random_normal(&r, vd, rn);
  correct_normal(rn, vd, ivl);
  float rh[5][4] = {{normal[0], normal[1], normal[2], depth},
                    {nn[0], nn[1], nn[2], depth},
                    {normal[0], normal[1], normal[2], ndepth},
                    {rn[0], rn[1], rn[2], depth},
                    {normal[0], normal[1], normal[2], rdepth}};
  costs[0] = 0;
  if (mi != 0)
    for (int v = 0; v < N; ++v) M[0][v] = M[mi][v];
  for (int v = 0; v < N; ++v) costs[0] += vw[v] * M[0][v];
  const int nh = rand_depth ? 5 : 4;
  for (int h = 1; h < nh; ++h) {
    cost_vector(c, row, col, rh[h][3], rh[h], np, &pr, M[h], prior_weight(c, &pri, rh[h], rh[h][3], pr.rvar));
    float cs = 0;
    for (int v = 0; v < N; ++v) cs += vw[v] * M[h][v];
    costs[h] = cs;
  }
  mi = find_min_cost(costs, nh);
  if (mi != -1) {
    c->conf[pix] = costs[mi];
    c->depth[pix] = rh[mi][3];
    c->normal[pix] = rh[mi][0]; c->normal[WH + pix] = rh[mi][1]; c->normal[2 * WH + pix] = rh[mi][2];
    for (int v = 0; v < N; ++v) c->cost[(size_t)v * WH + pix] = M[mi][v];
  }
}

/* LocalOptimization, kernel_functions.cu:2736-2931, for one pixel. */
static void local_opt_pixel(ctx_t* c, int row, int col, uint64_t sk) {
  const int W = c->W, H = c->H, N = c->N;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  rng_t r = rng_make(sk, (uint32_t)pix);
  float conf = c->conf[pix];
  float depth = c->depth[pix];
  float normal[3] = {c->normal[pix], c->normal[WH + pix], c->normal[2 * WH + pix]};
  const uint32_t sel = c->view_sel[pix];
  const float a1 = (float)DEG2RAD_D(4.0), a2 = (float)DEG2RAD_D(2.0);
  const float* iK = c->refiK;
  const float np[3] = {iK[0] * col + iK[1], iK[2] * row + iK[3], 1.0f};
  float m[3] = {normal[0], normal[1], normal[2]};
  float lo = depth, hi = depth;
  for (int i = 0; i < 4; ++i) {
    const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
    if (u < 0 || u >= W || v < 0 || v >= H) continue;
    const size_t q = (size_t)v * W + u;
    const float nd = c->depth[q];
    m[0] += c->normal[q]; m[1] += c->normal[WH + q]; m[2] += c->normal[2 * WH + q];
    if (nd <= lo) lo = nd;
    if (nd > hi) hi = nd;
  }
  const float inv_norm = 1.0f / sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  m[0] *= inv_norm; m[1] *= inv_norm; m[2] *= inv_norm;
  pixref_t pr;
  load_pixref(c, row, col, &pr);
  float M[5][SMVS_MAX_SRC];
  float hyp[5][4];
  int mi = -1;
  for (int it = 0; it < 5; ++it) {
    hyp[it][3] = rng_uniform(&r) * (hi - lo) + lo;
    perturb_normal_acmh(m, hyp[it], a1, a2, &r);
    float mconf = 0, mw = 0;
    for (int v = 0; v < N; ++v) {
      if (!((sel >> v) & 1u)) continue;
      float cost = ncc_cost(c, v, row, col, hyp[it][3], hyp[it], &pr);
      if (c->geom) cost += c->geom_reg * geom_cost(c, v, (float)row, (float)col, hyp[it][3], np, c->refK);
      M[it][v] = cost;
      mconf += cost;
      mw += 1;
    }
    if (mw <= 0) return;
    mconf /= mw;
    if (mconf < conf) {
      conf = mconf;
      depth = hyp[it][3];
      normal[0] = hyp[it][0]; normal[1] = hyp[it][1]; normal[2] = hyp[it][2];
      mi = it;
    }
  }
  if (mi != -1) {
    c->conf[pix] = conf;
    c->depth[pix] = depth;
    c->normal[pix] = normal[0]; c->normal[WH + pix] = normal[1]; c->normal[2 * WH + pix] = normal[2];
    for (int v = 0; v < N; ++v) {
      if ((sel >> v) & 1u) {
        c->cost[(size_t)v * WH + pix] = M[mi][v];
      } else {
        float cost = ncc_cost(c, v, row, col, depth, normal, &pr);
        /* [quirk] :2916-2919 passes the inverse intrinsics where K is expected */
        if (c->geom) cost += c->geom_reg * geom_cost(c, v, (float)row, (float)col, depth, np, c->refiK);
        c->cost[(size_t)v * WH + pix] = cost;
      }
    }
  }
}

static void half_sweep(ctx_t* c, int colour, int row_begin, int row_end, int local, float th_mc,
                       uint64_t sk) {
  /* The pixels of one colour are independent: parallel over pixels (not rows),
   * so that a band of a few rows still keeps every thread busy. */
  const int W = c->W, half = (W + 1) / 2;
  const long n = (long)(row_end - row_begin) * half;
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    const int row = row_begin + (int)(i / half);
    const int col = 2 * (int)(i % half) + ((row + colour) & 1);
    if (col >= W) continue;
    if (local) local_opt_pixel(c, row, col, sk);
    else sweep_pixel(c, row, col, th_mc, sk);
  }
}


/* ComputeCurvatureMap, kernel_functions.cu:1603-1653. */
static void curvature_map(const ctx_t* c, uint16_t* out) {
  const int W = c->W, H = c->H;
  const size_t WH = (size_t)W * H;
#pragma omp parallel for schedule(static)
  for (int row = 0; row < H; ++row)
    for (int col = 0; col < W; ++col) {
      const size_t pix = (size_t)row * W + col;
      float gx = 0, gy = 0;
      for (int dr = -1; dr <= 1; ++dr)
        for (int dc = -1; dc <= 1; ++dc) {
          const float color = ref_at(c, row + dr, col + dc);
          gx += color * kScharrX[dr + 1][dc + 1];
          gy += color * kScharrY[dr + 1][dc + 1];
        }
      const float grad = sqrtf(gx * gx + gy * gy);
      const int x0 = col - 2 > 0 ? col - 2 : 0, x1 = col + 2 < W - 1 ? col + 2 : W - 1;
      const int y0 = row - 2 > 0 ? row - 2 : 0, y1 = row + 2 < H - 1 ? row + 2 : H - 1;
      const float n0 = c->normal[pix], n1 = c->normal[WH + pix], n2 = c->normal[2 * WH + pix];
      float ang[24];
      int cnt = 0;
      for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
          if (y == row && x == col) continue;
          const size_t q = (size_t)y * W + x;
          ang[cnt++] = acosf(n0 * c->normal[q] + n1 * c->normal[WH + q] + n2 * c->normal[2 * WH + q]);
        }
      out[pix] = (uint16_t)fminf(grad * 10000.f, 32767.f);
      float med = 3.14159265358979323846f * 10000.0f;
      if (cnt > 0) {
        for (int i = 0; i < cnt - 1; ++i)
          for (int j = 0; j < cnt - 1 - i; ++j)
            if (ang[j] > ang[j + 1]) { float t = ang[j]; ang[j] = ang[j + 1]; ang[j + 1] = t; }
        med = ang[cnt / 2] * 10000.0f;
      }
      out[WH + pix] = (med != med) ? 0 : (uint16_t)fminf(fmaxf(med, 0.f), 65535.f);
    }
}

/* ComputeGeomGradientMap (kernel_functions.cu:3095-3120; 0 where depth <= 0)
 * + MedianFilter via Black/RedPixelFilter (:3122-3280). */
static void median_filter(ctx_t* c, float diff_thres) {
  const int W = c->W, H = c->H;
  const size_t WH = (size_t)W * H;
  float* gg = (float*)malloc(sizeof(float) * WH);
  if (!gg) return;
#pragma omp parallel for schedule(static)
  for (int row = 0; row < H; ++row)
    for (int col = 0; col < W; ++col) {
      const size_t pix = (size_t)row * W + col;
      const float d = c->depth[pix];
      if (d <= 0) { gg[pix] = 0; continue; }
      float gx = 0, gy = 0;
      for (int dr = -1; dr <= 1; ++dr)
        for (int dc = -1; dc <= 1; ++dc) {
          const int nr = row + dr, nc = col + dc;
          if (nr < 0 || nr >= H || nc < 0 || nc >= W) continue;
          const float diff = fabsf(c->depth[(size_t)nr * W + nc] - d) / d;
          gx += diff * kScharrX[dr + 1][dc + 1];
          gy += diff * kScharrY[dr + 1][dc + 1];
        }
      gg[pix] = sqrtf(gx * gx + gy * gy);
    }
  const float grad_thres = 1.4f * diff_thres;
  static const int dirs[8][2] = {{-2, 1}, {-1, 2}, {1, 2}, {2, 1}, {2, -1}, {1, -2}, {-1, -2}, {-2, -1}};
  for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
    for (int row = 0; row < H; ++row)
      for (int col = ((row + colour) & 1); col < W; col += 2) {
        const size_t pix = (size_t)row * W + col;
        float dep[17], nx[17], ny[17], nz[17];
        const float grad = gg[pix], cd = c->depth[pix], icd = 1.0f / cd;
        int idx = 0;
        dep[0] = cd; nx[0] = c->normal[pix]; ny[0] = c->normal[WH + pix]; nz[0] = c->normal[2 * WH + pix];
        idx = 1;
        int cand[16][2], nc = 0;
        for (int i = 0; i < 2; ++i) {
          const int o = 2 * i + 1;
          if (row - o >= 0) { cand[nc][0] = row - o; cand[nc][1] = col; nc++; }
          if (row + o < H) { cand[nc][0] = row + o; cand[nc][1] = col; nc++; }
          if (col - o >= 0) { cand[nc][0] = row; cand[nc][1] = col - o; nc++; }
          if (col + o < W) { cand[nc][0] = row; cand[nc][1] = col + o; nc++; }
        }
        for (int i = 0; i < 8; ++i) {
          const int r2 = row + dirs[i][0], c2 = col + dirs[i][1];
          if (r2 >= 0 && r2 < H && c2 >= 0 && c2 < W) { cand[nc][0] = r2; cand[nc][1] = c2; nc++; }
        }
        for (int k = 0; k < nc; ++k) {
          const size_t q = (size_t)cand[k][0] * W + cand[k][1];
          dep[idx] = c->depth[q];
          const float diff = fabsf(dep[idx] - cd) * icd;
          if (grad < grad_thres || (grad >= grad_thres && diff < diff_thres)) {
            nx[idx] = c->normal[q]; ny[idx] = c->normal[WH + q]; nz[idx] = c->normal[2 * WH + q];
            idx++;
          }
        }
        float* arrs[4] = {dep, nx, ny, nz};
        for (int a = 0; a < 4; ++a) {
          float* v = arrs[a];
          for (int i = 0; i < idx - 1; ++i)
            for (int j = 0; j < idx - 1 - i; ++j)
              if (v[j] > v[j + 1]) { float t = v[j]; v[j] = v[j + 1]; v[j + 1] = t; }
        }
        const int nth = idx >> 1;
        const float inv = 1.0f / sqrtf(nx[nth] * nx[nth] + ny[nth] * ny[nth] + nz[nth] * nz[nth]);
        c->depth[pix] = dep[nth];
        c->normal[pix] = nx[nth] * inv; c->normal[WH + pix] = ny[nth] * inv; c->normal[2 * WH + pix] = nz[nth] * inv;
      }
  }
  free(gg);
}

/* FilterDepthMap, kernel_functions.cu:3282-3354, launched black then red
 * (patch_match_cuda.cu:1015-1038) over rows r with r/2 < ceil((H/2)/16)*16. */
static void conf_filter(ctx_t* c, float depth_thres, float conf_thres) {
  const int W = c->W, H = c->H;
  const size_t WH = (size_t)W * H;
  const int row_pairs = ((H / 2) + 15) / 16 * 16;
  for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
    for (int row = 0; row < H; ++row) {
      if ((row >> 1) >= row_pairs) continue;
      for (int col = ((row + colour) & 1); col < W; col += 2) {
        const size_t pix = (size_t)row * W + col;
        const float d = c->depth[pix];
        if (d <= 0) continue;
        const float n[3] = {c->normal[pix], c->normal[WH + pix], c->normal[2 * WH + pix]};
        const float conf = c->conf[pix];
        const float* iK = c->refiK;
        const float pt[3] = {d * (iK[0] * col + iK[1]), d * (iK[2] * row + iK[3]), d};
        int good = 0;
        for (int i = 0; i < 4; ++i) {
          const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
          if (u < 0 || u >= W || v < 0 || v >= H) continue;
          const size_t q = (size_t)v * W + u;
          const float nd = c->depth[q];
          const float nn[3] = {c->normal[q], c->normal[WH + q], c->normal[2 * WH + q]};
          const float nconf = c->conf[q];
          const float np[3] = {nd * (iK[0] * u + iK[1]), nd * (iK[2] * v + iK[3]), nd};
          const float d1 = fabsf((pt[0] - np[0]) * n[0] + (pt[1] - np[1]) * n[1] + (pt[2] - np[2]) * n[2]);
          const float d2 = fabsf((pt[0] - np[0]) * nn[0] + (pt[1] - np[1]) * nn[1] + (pt[2] - np[2]) * nn[2]);
          if ((conf < conf_thres && d1 / d < depth_thres) || (nconf < conf_thres && d2 / nd < depth_thres)) good++;
        }
        if (good < 2) {
          c->depth[pix] = 0; c->normal[pix] = 0; c->normal[WH + pix] = 0; c->normal[2 * WH + pix] = 0;
          c->conf[pix] = 0;
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Set-up and public entry points                                             */
/* ------------------------------------------------------------------------ */
static int supported_window(int R, int S) { /* dispatcher, kernel_functions.cu:1343-1400 */
  return (S == 1 && (R == 3 || R == 5 || R == 7)) || (S == 2 && (R == 3 || R == 4 || R == 5 || R == 7));
}

static float pixel_value(const smvs_view* v, int x, int y) {
  const size_t stride = v->row_stride ? v->row_stride
                                      : (size_t)v->width * (v->pixel_format == SMVS_PIX_U8 ? 1 : 4);
  const char* rowp = (const char*)v->pixels + stride * (size_t)y;
  if (v->pixel_format == SMVS_PIX_U8) return (float)((const uint8_t*)rowp)[x];
  return ((const float*)rowp)[x];
}
static inline float quantise_u8(float g) {
  float q = nearbyintf(g);
  return q < 0 ? 0 : (q > 255 ? 255 : q);
}

static void ctx_free(ctx_t* c) {
  free(c->poses); free(c->ref); free(c->ref_sum); free(c->ref_sqsum); free(c->grad);
  for (int i = 0; i < SMVS_MAX_SRC; ++i) { free(c->src[i]); }
  free(c->depth); free(c->normal); free(c->conf); free(c->cost); free(c->view_sel);
}

static int ctx_init(ctx_t* c, const smvs_options* o, const smvs_problem* p, int need_state) {
  memset(c, 0, sizeof(*c));
  if (!o || !p || p->memory != SMVS_MEM_HOST) return SMVS_EINVAL;
  if (p->num_src < 1 || p->num_src > SMVS_MAX_SRC) return SMVS_EINVAL;
  if (!supported_window(o->window_radius, o->window_step)) return SMVS_EINVAL;
  if (o->thk < 1 || o->thk > 4) return SMVS_EINVAL;
  c->W = p->ref.width; c->H = p->ref.height; c->N = p->num_src;
  c->R = o->window_radius; c->S = o->window_step;
  const float ss = (float)o->sigma_spatial, sc = (float)o->sigma_color;
  c->sn = 1.0f / (2.0f * ss * ss);
  c->cn = 1.0f / (2.0f * sc * sc);
  c->sigma_s = o->sigma_spatial; c->sigma_c = o->sigma_color;
  c->depth_min = (float)o->depth_min; c->depth_max = (float)o->depth_max;
  c->num_samples = o->num_samples;
  c->thk = o->thk < c->N ? o->thk : c->N; /* :949-950 */
  c->num_good = o->num_good_hypothesis; c->num_bad = o->num_bad_hypothesis;
  c->random_opt = o->random_optimization; c->local_opt = o->local_optimization;
  c->geom = o->geom_consistency; c->num_iter = o->num_iterations;
  c->geom_reg = (float)o->geom_consistency_regularizer; c->geom_max = (float)o->geom_consistency_max_cost;
  c->rand_depth_ratio = o->random_depth_ratio;
  c->rand_a1 = o->random_angle1_range; c->rand_a2 = o->random_angle2_range;
  c->init_mc = (float)o->init_ncc_matching_cost; c->max_mc = (float)o->max_ncc_matching_cost;
  c->alpha = (float)o->alpha; c->beta = (float)o->beta;
  c->seed = o->random_seed;
  c->src_half = (o->image_storage == SMVS_STORE_F16);
  const size_t WH = (size_t)c->W * c->H;
  c->poses = (float*)malloc(sizeof(float) * SMVS_POSE_FLOATS * c->N);
  c->ref = (float*)malloc(sizeof(float) * WH);
  c->ref_sum = (float*)malloc(sizeof(float) * WH);
  c->ref_sqsum = (float*)malloc(sizeof(float) * WH);
  c->grad = (float*)malloc(sizeof(float) * WH);
  if (!c->poses || !c->ref || !c->ref_sum || !c->ref_sqsum || !c->grad) return SMVS_ENOMEM;
  build_poses(p, c->refK, c->refiK, c->poses);
  /* The reference image is uint8 and read normalised (patch_match_cuda.cu:132-147). */
  for (int y = 0; y < c->H; ++y)
    for (int x = 0; x < c->W; ++x) c->ref[(size_t)y * c->W + x] = quantise_u8(pixel_value(&p->ref, x, y)) / 255.0f;
  for (int i = 0; i < c->N; ++i) {
    const smvs_view* s = &p->src[i];
    c->sw[i] = s->width; c->sh[i] = s->height;
    c->src[i] = (float*)malloc(sizeof(float) * (size_t)s->width * s->height);
    if (!c->src[i]) return SMVS_ENOMEM;
    for (int y = 0; y < s->height; ++y)
      for (int x = 0; x < s->width; ++x) {
        float g = pixel_value(s, x, y);
        float val;
        if (o->image_storage == SMVS_STORE_U8) val = quantise_u8(g) / 255.0f;
        else if (o->image_storage == SMVS_STORE_F16) val = round_to_half(g / 255.0f);
        else val = g / 255.0f;
        c->src[i][(size_t)y * s->width + x] = val;
      }
    c->sdepth[i] = (float*)s->depth; /* borrowed */
    if (c->geom && !s->depth) return SMVS_EINVAL;
  }
  prep_ref(c);
  if (need_state) {
    c->depth = (float*)malloc(sizeof(float) * WH);
    c->normal = (float*)malloc(sizeof(float) * 3 * WH);
    c->conf = (float*)malloc(sizeof(float) * WH);
    c->cost = (float*)malloc(sizeof(float) * c->N * WH);
    c->view_sel = (uint32_t*)malloc(sizeof(uint32_t) * WH);
    if (!c->depth || !c->normal || !c->conf || !c->cost || !c->view_sel) return SMVS_ENOMEM;
  }
  return SMVS_OK;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* PatchMatchACMMCuda::Run, patch_match_cuda.cu:748-1057 (photometric or
 * geometric pass, then curvature, median filter, confidence filter, mask). */
int orc_run(const smvs_options* o, const smvs_problem* p, int row_begin, int row_end, orc_outputs* out) {
  ctx_t c;
  int st = ctx_init(&c, o, p, 1);
  if (st != SMVS_OK) { ctx_free(&c); return st; }
  if (o->has_prior_depth && o->propagate_depth) { ctx_free(&c); return SMVS_EINVAL; }
  if (o->propagate_depth && (o->init_depth_random || o->geom_consistency)) { ctx_free(&c); return SMVS_EINVAL; }
  if (o->has_prior_depth && (!p->ref.depth || !p->ref.normal)) { ctx_free(&c); return SMVS_EINVAL; }
  if (!o->init_depth_random && (!p->ref.depth || !p->ref.normal)) { ctx_free(&c); return SMVS_EINVAL; }
  const size_t WH0 = (size_t)c.W * c.H;
  float *pdepth = NULL, *pnormal = NULL, *pprior = NULL;
  const float* init_depth = p->ref.depth;
  const float* init_normal = p->ref.normal;
  if (o->has_prior_depth) { /* InitPriorDepthAndNormalInfo, patch_match_cuda.cu:715-746 */
    c.prior_mode = 1;
    c.prior_depth = p->ref.depth;
    c.prior_normal = p->ref.normal;
    c.prior_wgt = p->ref_prior_wgt;
  } else if (o->propagate_depth) { /* patch_match_cuda.cu:603-659 */
    pdepth = (float*)malloc(sizeof(float) * WH0);
    pnormal = (float*)malloc(sizeof(float) * 3 * WH0);
    pprior = (float*)malloc(sizeof(float) * WH0);
    if (!pdepth || !pnormal || !pprior) { free(pdepth); free(pnormal); free(pprior); ctx_free(&c); return SMVS_ENOMEM; }
    memcpy(pdepth, p->ref.depth, sizeof(float) * WH0);
    memcpy(pnormal, p->ref.normal, sizeof(float) * 3 * WH0);
    st = orc_propagate_init(c.W, c.H, c.N, c.refK, c.refiK, c.poses, p->src, pdepth, pnormal, pprior);
    if (st != SMVS_OK) { free(pdepth); free(pnormal); free(pprior); ctx_free(&c); return st; }
    c.prior_mode = 2;
    c.prior_depth = pprior;
    init_depth = pdepth;
    init_normal = pnormal;
  }
  init_workspace(&c, o->init_depth_random, init_depth, init_normal, (float)o->depth_min, (float)o->depth_max);
  free(pdepth);
  free(pnormal);
  int rb = 0, re = c.H;
  if (row_end > row_begin) { rb = row_begin < 0 ? 0 : row_begin; re = row_end > c.H ? c.H : row_end; }
  {
    /* A band run scores the initial hypotheses of the band and of the rows
     * its sweeps read (neighbour samples reach 21 rows, kernel_functions.cu:
     * 27-44); other rows keep conf 0 and are never read. */
    const int margin = 24;
    const int cb = (rb == 0 && re == c.H) ? 0 : (rb - margin < 0 ? 0 : rb - margin);
    const int ce = (rb == 0 && re == c.H) ? c.H : (re + margin > c.H ? c.H : re + margin);
    if (cb > 0 || ce < c.H) memset(c.conf, 0, sizeof(float) * (size_t)c.W * c.H);
    init_conf(&c, cb, ce);
  }
  for (int iter = 0; iter < c.num_iter; ++iter) {
    const float th_mc = c.init_mc * expf(-(float)(iter * iter) / c.alpha); /* :778-779 */
    half_sweep(&c, 0, rb, re, 0, th_mc, stage_key(c.seed, stage_sweep(iter, 0)));
    half_sweep(&c, 1, rb, re, 0, th_mc, stage_key(c.seed, stage_sweep(iter, 1)));
    if (c.local_opt && iter > 2 && !o->has_prior_depth) { /* :861-880 */
      half_sweep(&c, 0, rb, re, 1, th_mc, stage_key(c.seed, stage_local(iter, 0)));
      half_sweep(&c, 1, rb, re, 1, th_mc, stage_key(c.seed, stage_local(iter, 1)));
    }
  }
  uint16_t* curv = NULL;
  if (o->est_curvature && c.geom) { /* patch_match_cuda.cu:985-989 */
    curv = (uint16_t*)malloc(sizeof(uint16_t) * 2 * (size_t)c.W * c.H);
    if (curv) curvature_map(&c, curv);
  }
  if (o->median_filter) median_filter(&c, o->depth_diff_threshold);                 /* :991-1008 */
  if (o->filter && o->conf_filter) conf_filter(&c, o->depth_diff_threshold, o->conf_threshold); /* :1015-1038 */
  if (p->ref_mask) { /* MaskDepthMapKernel :3080-3093 ([quirk] last row/col untouched) */
    for (int y = 0; y < c.H - 1; ++y)
      for (int x = 0; x < c.W - 1; ++x)
        if (p->ref_mask[(size_t)y * c.W + x] == 0) c.depth[(size_t)y * c.W + x] = 0.0f;
  }
  const size_t WH = (size_t)c.W * c.H;
  if (out) {
    if (out->depth) memcpy(out->depth, c.depth, sizeof(float) * WH);
    if (out->normal) memcpy(out->normal, c.normal, sizeof(float) * 3 * WH);
    if (out->conf) memcpy(out->conf, c.conf, sizeof(float) * WH);
    if (out->cost) memcpy(out->cost, c.cost, sizeof(float) * c.N * WH);
    if (out->view_sel) memcpy(out->view_sel, c.view_sel, sizeof(uint32_t) * WH);
    if (out->grad) memcpy(out->grad, c.grad, sizeof(float) * WH);
    if (out->ref_sum) memcpy(out->ref_sum, c.ref_sum, sizeof(float) * WH);
    if (out->ref_sqsum) memcpy(out->ref_sqsum, c.ref_sqsum, sizeof(float) * WH);
    if (out->poses) memcpy(out->poses, c.poses, sizeof(float) * SMVS_POSE_FLOATS * c.N);
    if (out->curvature && curv) memcpy(out->curvature, curv, sizeof(uint16_t) * 2 * WH);
  }
  free(curv);
  free(pprior);
  ctx_free(&c);
  return SMVS_OK;
}

/* ComputeGeomConsistencyCost (texture form), kernel_functions.cu:570-633 — the
 * same arithmetic as the shared-memory form with K = ref_K. */
/* FilterDepthMapsKernel, kernel_functions.cu:3356-3410; RunFilter(false),
 * patch_match_cuda.cu:1075-1108. */
int orc_run_filter(const smvs_options* o, const smvs_problem* p, float* depth_out) {
  ctx_t c;
  smvs_options oo = *o;
  oo.geom_consistency = 1;
  int st = ctx_init(&c, &oo, p, 0);
  if (st != SMVS_OK) { ctx_free(&c); return st; }
  if (!p->ref.depth) { ctx_free(&c); return SMVS_EINVAL; }
  int min_cons = o->filter_min_num_consistent < c.N ? o->filter_min_num_consistent : c.N;
  const float fmax = (float)o->filter_geom_consistency_max_cost;
#pragma omp parallel for schedule(static)
  for (int row = 0; row < c.H; ++row)
    for (int col = 0; col < c.W; ++col) {
      const size_t pix = (size_t)row * c.W + col;
      const float d = p->ref.depth[pix];
      if (d < 1e-6f) { depth_out[pix] = 0.0f; continue; }
      const float np[3] = {c.refiK[0] * col + c.refiK[1], c.refiK[2] * row + c.refiK[3], 1.0f};
      int good = 0;
      for (int v = 0; v < c.N; ++v)
        if (geom_cost(&c, v, (float)row, (float)col, d, np, c.refK) <= fmax) good++;
      depth_out[pix] = (good < min_cons) ? 0.0f : d;
    }
  ctx_free(&c);
  return SMVS_OK;
}

/* FP64 evaluation of ComputeNCCCost at one pixel (direct homography per tap,
 * exact bilinear weights, exact exp/sqrt). */
static double ncc_cost_f64(const ctx_t* c, int v, int row, int col, double depth, const float nf[3]) {
  const float* pose = c->poses + (size_t)v * SMVS_POSE_FLOATS;
  double K[4], Rm[9], T[3], iK[4], n[3] = {nf[0], nf[1], nf[2]};
  for (int k = 0; k < 4; ++k) { K[k] = pose[k]; iK[k] = c->refiK[k]; }
  for (int k = 0; k < 9; ++k) Rm[k] = pose[4 + k];
  for (int k = 0; k < 3; ++k) T[k] = pose[13 + k];
  /* H = Ks (R + T n^T / d) Kr^-1 with d = depth * n . Kr^-1 x (the reference's
   * sign convention, kernel_functions.cu:446-458). */
  const double dist = depth * (n[0] * (iK[0] * col + iK[1]) + n[1] * (iK[2] * row + iK[3]) + n[2]);
  double A[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i * 3 + j] = Rm[i * 3 + j] + T[i] * n[j] / dist;
  const double Ks[9] = {K[0], 0, K[1], 0, K[2], K[3], 0, 0, 1};
  const double Ki[9] = {iK[0], 0, iK[1], 0, iK[2], iK[3], 0, 0, 1};
  double KA[9], Hd[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += Ks[i * 3 + k] * A[k * 3 + j];
      KA[i * 3 + j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += KA[i * 3 + k] * Ki[k * 3 + j];
      Hd[i * 3 + j] = s;
    }
  const double z0 = Hd[6] * col + Hd[7] * row + Hd[8];
  const double u0 = (Hd[0] * col + Hd[1] * row + Hd[2]) / z0, v0 = (Hd[3] * col + Hd[4] * row + Hd[5]) / z0;
  const int ui = (u0 != u0) ? 0 : (int)fmax(fmin(u0, 2e9), -2e9), vi = (v0 != v0) ? 0 : (int)fmax(fmin(v0, 2e9), -2e9);
  if (ui < 0 || ui >= c->W || vi < 0 || vi >= c->H) return 2.0;
  const int R = c->R, S = c->S;
  const double center = c->ref[(size_t)row * c->W + col];
  const double sn = 1.0 / (2.0 * c->sigma_s * c->sigma_s);
  const double cn = 1.0 / (2.0 * c->sigma_c * c->sigma_c);
  double sw = 0, sr = 0, srr = 0, ss = 0, sss = 0, srs = 0;
  for (int dr = -R; dr <= R; dr += S)
    for (int dc = -R; dc <= R; dc += S) {
      const double x = col + dc, y = row + dr;
      const double z = Hd[6] * x + Hd[7] * y + Hd[8];
      const double su = (Hd[0] * x + Hd[1] * y + Hd[2]) / z, sv = (Hd[3] * x + Hd[4] * y + Hd[5]) / z;
      const double rc = ref_at(c, row + dr, col + dc);
      const double sc = tex_bilinear_f64(c->src[v], c->sw[v], c->sh[v], su + 0.5, sv + 0.5);
      const double w = exp(-(double)(dr * dr + dc * dc) * sn - (center - rc) * (center - rc) * cn);
      sw += w; sr += w * rc; srr += w * rc * rc; ss += w * sc; sss += w * sc * sc; srs += w * rc * sc;
    }
  /* Reference moments over the same window (the FilterKernel sums). */
  const double mr = sr / sw, vr = srr / sw - mr * mr;
  const double ms = ss / sw, vs = sss / sw - ms * ms;
  if (vr < 1e-5 || vs < 1e-5) return 2.0;
  const double val = 1.0 - (srs / sw - mr * ms) / sqrt(vr * vs);
  return fmax(0.0, fmin(2.0, val));
}

int orc_eval_costs(const smvs_options* o, const smvs_problem* p, int n_pix, const int* rows, const int* cols,
                   const float* depths, const float* normals, float* costs32, double* costs64) {
  ctx_t c;
  smvs_options oo = *o;
  oo.geom_consistency = 0;
  int st = ctx_init(&c, &oo, p, 0);
  if (st != SMVS_OK) { ctx_free(&c); return st; }
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n_pix; ++i) {
    pixref_t pr;
    const int row = rows[i], col = cols[i];
    if (row < 0 || row >= c.H || col < 0 || col >= c.W) continue;
    load_pixref(&c, row, col, &pr);
    for (int v = 0; v < c.N; ++v) {
      if (costs32) costs32[(size_t)i * c.N + v] = ncc_cost(&c, v, row, col, depths[i], normals + 3 * i, &pr);
      if (costs64) costs64[(size_t)i * c.N + v] = ncc_cost_f64(&c, v, row, col, depths[i], normals + 3 * i);
    }
  }
  ctx_free(&c);
  return SMVS_OK;
}
