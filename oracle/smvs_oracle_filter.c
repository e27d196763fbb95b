/*
 * smvs_oracle_filter.c — CPU oracle of the cross-view filter and deduplication.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of sensemap_b200/csrc/smvs_cross_filter.cu
 * and the CPU arm of its benchmark; the product never links or calls it.
 *
 * Restates CrossFilterCuda (SenseMap src/mvs/patch_match_cuda.cu:1111-1710) and
 * its kernels CrossFilterKernel / DeduplicFilterKernel / GetDeduplicDepthMapsLayer
 * (src/mvs/kernel_functions.cu:3561-3960) on the CPU, problem by problem in the
 * reference's order. Built with -ffp-contract=off: the same IEEE single-
 * precision operations, in the same order, as the CUDA unit (compiled with
 * -fmad=false, -prec-div=true, -prec-sqrt=true, -ftz=false), with fused
 * multiply-adds only where both write fmaf, so the two agree bit for bit.
 * Differences from the reference, shared with the CUDA kernels:
 *   - depth and normal maps are read with exact point sampling (texel
 *     floor(x + 0.5)) instead of the texture unit's fixed-point coordinates;
 *   - the reference is built with --use_fast_math (approximate reciprocal,
 *     division and square root); both here use IEEE operations;
 *   - a view marked ref_flag that no problem refined reads an all-zero map
 *     (the reference reads an uninitialised 1x1 buffer, :1270-1276).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

#include "smvs_oracle.h"
#include "orc_pose.h"

#define DEG2RAD_F(deg) ((deg) * 0.0174532925199432) /* kernel_functions.h:39 */
#define VIS_KEEP 0x80000000u

/* NormalMap::Encode, normal_map.cc:159-181 (same expression types). */
static uint32_t encode_normal(float n0, float n1, float n2) {
  const float s = (float)((1 - n0) * 0.5);
  const float m = 1.0f / sqrtf(1 - s);
  float q1 = (float)(n1 * 0.5 * m), q2 = (float)(n2 * 0.5 * m);
  /* std::min(0.999999f, std::max(q, -0.999999f)): a NaN clamps to +0.999999 */
  q1 = q1 < -0.999999f ? -0.999999f : q1;
  q1 = q1 < 0.999999f ? q1 : 0.999999f;
  q2 = q2 < -0.999999f ? -0.999999f : q2;
  q2 = q2 < 0.999999f ? q2 : 0.999999f;
  const uint32_t iq1 = (uint32_t)((q1 + 1) * 32767.f), iq2 = (uint32_t)((q2 + 1) * 32767.f);
  return (iq1 << 16) | iq2;
}

/* The in-kernel decode, kernel_functions.cu:3592-3601 (decode_factor = 32767, :9). */
static void decode_normal(uint32_t code, float n[3]) {
  const uint32_t iq1 = code >> 16, iq2 = code & 0x0000ffffu;
  const float q1 = (float)iq1 / 32767.f - 1, q2 = (float)iq2 / 32767.f - 1;
  const float s = fmaf(q1, q1, q2 * q2);
  n[0] = (float)(1.0 - 2.0 * s);
  n[1] = 2 * q1 * sqrtf(1 - s);
  n[2] = 2 * q2 * sqrtf(1 - s);
}

static int check_set(const smvs_filter_view* views, int nv, const smvs_filter_problem* probs, int np) {
  if (!views || nv < 1 || (np > 0 && !probs)) return SMVS_EINVAL;
  for (int v = 0; v < nv; ++v)
    if (views[v].width < 1 || views[v].height < 1 || !views[v].depth) return SMVS_EINVAL;
  for (int p = 0; p < np; ++p) {
    if (probs[p].ref < 0 || probs[p].ref >= nv || probs[p].num_src < 0 || probs[p].num_src > SMVS_CROSS_MAX_SRC)
      return SMVS_EINVAL;
    for (int i = 0; i < probs[p].num_src; ++i)
      if (probs[p].src[i] < 0 || probs[p].src[i] >= nv || probs[p].src[i] == probs[p].ref) return SMVS_EINVAL;
  }
  return SMVS_OK;
}

/* InitTransforms (:1320-1407): the reference view's K and the source pose
 * records, without source scaling. */
static void problem_poses(const smvs_filter_view* views, const smvs_filter_problem* pr, float refK[4],
                          float refiK[4], float* poses) {
  smvs_view ref, src[SMVS_CROSS_MAX_SRC];
  memset(&ref, 0, sizeof(ref));
  memset(src, 0, sizeof(src));
  const smvs_filter_view* rv = &views[pr->ref];
  memcpy(ref.K, rv->K, sizeof(ref.K)); memcpy(ref.R, rv->R, sizeof(ref.R)); memcpy(ref.T, rv->T, sizeof(ref.T));
  for (int i = 0; i < pr->num_src; ++i) {
    const smvs_filter_view* sv = &views[pr->src[i]];
    memcpy(src[i].K, sv->K, sizeof(src[i].K)); memcpy(src[i].R, sv->R, sizeof(src[i].R));
    memcpy(src[i].T, sv->T, sizeof(src[i].T));
    src[i].scale = 1.0f;
  }
  smvs_problem q;
  memset(&q, 0, sizeof(q));
  q.ref = ref;
  q.src = src;
  q.num_src = pr->num_src;
  build_poses(&q, refK, refiK, poses);
}

/* Projection into a source view and back (kernel_functions.cu:3627-3673 and
 * :3822-3868, the same expressions in both kernels). */
/* a . x + t with explicit fused multiply-adds: the one rounding order the CUDA
 * kernels use too (the reference's fast-math build contracts these sums). */
static inline float affine3(const float a[3], const float x[3], float t) {
  return fmaf(a[0], x[0], fmaf(a[1], x[1], fmaf(a[2], x[2], t)));
}
static inline float dot3f(const float a[3], const float b[3]) { return fmaf(a[0], b[0], fmaf(a[1], b[1], a[2] * b[2])); }

static inline void project(const float* pose, const float X[3], float* scol, float* srow) {
  const float* P = pose + 19;
  const float ifz = 1.0f / affine3(P + 8, X, P[11]);
  *scol = ifz * affine3(P, X, P[3]);
  *srow = ifz * affine3(P + 4, X, P[7]);
}

/* Point sample at (x + 0.5, y + 0.5) with border zero: texel floor(x + 0.5). */
static inline int texel(float scol, float srow, int w, int h, int* sx, int* sy) {
  const float fx = floorf(scol + 0.5f), fy = floorf(srow + 0.5f);
  if (!(fx >= 0.0f && fx < (float)w && fy >= 0.0f && fy < (float)h)) return 0;
  *sx = (int)fx;
  *sy = (int)fy;
  return 1;
}

static inline float back_project(const float* pose, const float refK[4], float scol, float srow, float sd,
                                 int col, int row, float* err) {
  const float* iP = pose + 31;
  const float x[3] = {scol * sd, srow * sd, sd};
  const float bx = affine3(iP, x, iP[3]);
  const float by = affine3(iP + 4, x, iP[7]);
  const float bz = affine3(iP + 8, x, iP[11]);
  const float ibz = 1.0f / bz;
  const float bcol = ibz * fmaf(refK[0], bx, refK[1] * bz);
  const float brow = ibz * fmaf(refK[2], by, refK[3] * bz);
  const float dc = (float)col - bcol, dr = (float)row - brow;
  *err = sqrtf(fmaf(dc, dc, dr * dr));
  return bz;
}

static inline void bubble_sort(float* v, int n) { /* BubbleSort, utils.h:205-221 */
  for (int i = 0; i < n - 1; ++i)
    for (int j = 0; j < n - 1 - i; ++j)
      if (v[j] > v[j + 1]) { const float t = v[j]; v[j] = v[j + 1]; v[j + 1] = t; }
}

int orc_cross_filter_run(const smvs_options* o, const smvs_filter_view* views, int nv,
                         const smvs_filter_problem* probs, int np, float* const* refined) {
  if (!o || !refined) return SMVS_EINVAL;
  int st = check_set(views, nv, probs, np);
  if (st) return st;
  for (int p = 0; p < np; ++p) {
    if (probs[p].num_src < 1) continue;
    if (!views[probs[p].ref].normal || !refined[probs[p].ref]) return SMVS_EINVAL;
    for (int i = 0; i < probs[p].num_src; ++i)
      if (!views[probs[p].src[i]].normal) return SMVS_EINVAL;
  }
  /* InitNormalMaps (:1205-1258): every map encoded once. */
  uint32_t** codes = (uint32_t**)calloc((size_t)nv, sizeof(uint32_t*));
  if (!codes) return SMVS_ENOMEM;
  for (int v = 0; v < nv; ++v) {
    if (!views[v].normal) continue;
    const size_t WH = (size_t)views[v].width * views[v].height;
    codes[v] = (uint32_t*)malloc(sizeof(uint32_t) * WH);
    if (!codes[v]) { st = SMVS_ENOMEM; goto done; }
    const float* n = views[v].normal;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < WH; ++k) codes[v][k] = encode_normal(n[k], n[WH + k], n[2 * WH + k]);
  }
  const float fmax_err = (float)o->filter_geom_consistency_max_cost;
  const float thr = o->depth_diff_threshold;
  const float thr2 = thr * thr;
  const float max_view_cos = cosf((float)DEG2RAD_F(100));
  const float max_cos = cosf((float)DEG2RAD_F((float)o->max_normal_error));
  for (int p = 0; p < np; ++p) {
    const smvs_filter_problem* pr = &probs[p];
    if (pr->num_src < 1) continue; /* :1504-1506 */
    const smvs_filter_view* rv = &views[pr->ref];
    const int W = rv->width, H = rv->height, N = pr->num_src;
    const int min_cons = o->filter_min_num_consistent < N ? o->filter_min_num_consistent : N;
    float refK[4], refiK[4], poses[SMVS_CROSS_MAX_SRC * SMVS_POSE_FLOATS];
    problem_poses(views, pr, refK, refiK, poses);
    float* out = refined[pr->ref];
#pragma omp parallel for schedule(static)
    for (int row = 0; row < H; ++row)
      for (int col = 0; col < W; ++col) {
        const size_t pix = (size_t)row * W + col;
        const float depth = rv->depth[pix];
        if ((double)depth < 1e-6 || col < 3 || col > W - 3 || row < 3 || row > H - 3) { out[pix] = 0.0f; continue; }
        float rn[3];
        decode_normal(codes[pr->ref][pix], rn);
        float vr[3] = {fmaf(refiK[0], (float)col, refiK[1]), fmaf(refiK[2], (float)row, refiK[3]), 1.0f};
        const float X[3] = {depth * vr[0], depth * vr[1], depth};
        const float nvr = sqrtf(dot3f(vr, vr));
        vr[0] /= nvr; vr[1] /= nvr; vr[2] /= nvr;
        if (dot3f(rn, vr) >= max_view_cos) { out[pix] = 0.0f; continue; }
        float depths[SMVS_CROSS_MAX_SRC + 1];
        int good = 0;
        depths[0] = depth;
        for (int i = 0; i < N; ++i) {
          const float* pose = poses + (size_t)i * SMVS_POSE_FLOATS;
          const smvs_filter_view* sv = &views[pr->src[i]];
          float scol, srow;
          project(pose, X, &scol, &srow);
          int sx, sy;
          float sd = 0.0f;
          uint32_t scode = 0;
          if (texel(scol, srow, sv->width, sv->height, &sx, &sy)) {
            const size_t q = (size_t)sy * sv->width + sx;
            sd = sv->depth[q];
            scode = codes[pr->src[i]][q];
          }
          if ((double)sd < 1e-4) continue;
          float err;
          const float bz = back_project(pose, refK, scol, srow, sd, col, row, &err);
          if (err > fmax_err || (depth - bz) * (depth - bz) > depth * depth * thr2) continue;
          float sn[3];
          decode_normal(scode, sn);
          const float* R = pose + 4;  /* R^T n (kernel_functions.cu:3742-3747) */
          const float Rc0[3] = {R[0], R[3], R[6]}, Rc1[3] = {R[1], R[4], R[7]}, Rc2[3] = {R[2], R[5], R[8]};
          const float rs[3] = {dot3f(Rc0, sn), dot3f(Rc1, sn), dot3f(Rc2, sn)};
          if (dot3f(rn, rs) < max_cos) continue;
          depths[++good] = bz;
        }
        const int nth = (int)(good * 0.5);
        if (good >= min_cons) {
          bubble_sort(depths, good); /* sorts entries [0, good) of good + 1 (:3766) */
          out[pix] = depths[nth];
        } else {
          out[pix] = 0.0f;
        }
      }
  }
done:
  for (int v = 0; v < nv; ++v) free(codes[v]);
  free(codes);
  return st;
}

int orc_cross_filter_dedup(const smvs_options* o, const smvs_filter_view* views, int nv,
                           const smvs_filter_problem* probs, int np, const float* const* refined,
                           uint32_t* const* vis, float* const* delta) {
  if (!o || !vis || !delta) return SMVS_EINVAL;
  int st = check_set(views, nv, probs, np);
  if (st) return st;
  if (o->filter_min_num_consistent < 1) return SMVS_EINVAL;
  /* ResetDepthMaps (:1260-1318): refined maps for ref_flag views. */
  const float** dmap = (const float**)calloc((size_t)nv, sizeof(float*));
  float** zeros = (float**)calloc((size_t)nv, sizeof(float*));
  if (!dmap || !zeros) { free(dmap); free(zeros); return SMVS_ENOMEM; }
  for (int v = 0; v < nv; ++v) {
    const size_t WH = (size_t)views[v].width * views[v].height;
    if (!vis[v]) { st = SMVS_EINVAL; goto done; }
    for (size_t k = 0; k < WH; ++k) vis[v][k] = VIS_KEEP; /* FillGpuMat, :3930-3941 */
    if (views[v].ref_flag) {
      if (refined && refined[v]) {
        dmap[v] = refined[v];
      } else {
        zeros[v] = (float*)calloc(WH, sizeof(float));
        if (!zeros[v]) { st = SMVS_ENOMEM; goto done; }
        dmap[v] = zeros[v];
      }
    } else {
      dmap[v] = views[v].depth;
    }
  }
  for (int p = 0; p < np; ++p)
    if (probs[p].num_src >= 1 && !delta[probs[p].ref]) { st = SMVS_EINVAL; goto done; }
  const float fmax_err = (float)o->filter_geom_consistency_max_cost;
  const float thr = o->depth_diff_threshold;
  const float thr2 = thr * thr;
  for (int p = 0; p < np; ++p) {
    const smvs_filter_problem* pr = &probs[p];
    if (pr->num_src < 1) continue; /* :1568-1570 */
    const smvs_filter_view* rv = &views[pr->ref];
    const int W = rv->width, H = rv->height, N = pr->num_src;
    const int min_cons = o->filter_min_num_consistent < N ? o->filter_min_num_consistent : N;
    float refK[4], refiK[4], poses[SMVS_CROSS_MAX_SRC * SMVS_POSE_FLOATS];
    problem_poses(views, pr, refK, refiK, poses);
    const float* rd = dmap[pr->ref];
    uint32_t* rvis = vis[pr->ref];
    float* out = delta[pr->ref];
    memset(out, 0, sizeof(float) * (size_t)W * H);
#pragma omp parallel for schedule(static)
    for (int row = 0; row < H; ++row)
      for (int col = 0; col < W; ++col) {
        const size_t pix = (size_t)row * W + col;
        const float depth = rd[pix];
        if ((double)depth < 1e-6 || col < 3 || col > W - 3 || row < 3 || row > H - 3) { rvis[pix] = 0; continue; }
        /* [quirk] :3803 shifts by sizeof(uint32_t) - 1 = 3 bits, not 31 */
        if (!(rvis[pix] >> 3)) { rvis[pix] = 0; continue; }
        int good = 0, num_vis = 0;
        int idx[SMVS_CROSS_MAX_SRC + 1];
        float dd[SMVS_CROSS_MAX_SRC + 1];
        const float X[3] = {depth * fmaf(refiK[0], (float)col, refiK[1]), depth * fmaf(refiK[2], (float)row, refiK[3]),
                            depth};
        for (int i = 0; i < N; ++i) {
          const float* pose = poses + (size_t)i * SMVS_POSE_FLOATS;
          const int sv_i = pr->src[i];
          const smvs_filter_view* sv = &views[sv_i];
          float scol, srow;
          project(pose, X, &scol, &srow);
          int sx = 0, sy = 0;
          float sd = 0.0f;
          if (texel(scol, srow, sv->width, sv->height, &sx, &sy)) sd = dmap[sv_i][(size_t)sy * sv->width + sx];
          if (sd == 0.0f) continue;
          float err;
          const float bz = back_project(pose, refK, scol, srow, sd, col, row, &err);
          if (err > fmax_err || (depth - bz) * (depth - bz) > depth * depth * thr2) continue;
          ++good;
          dd[good - 1] = fabsf(bz - depth);
          idx[good] = i;
          /* visibility of the source at the same texel (:3900-3903) */
          if ((vis[sv_i][(size_t)sy * sv->width + sx] & VIS_KEEP) && sv->ref_flag) ++num_vis;
        }
        if (good < min_cons || num_vis > 0) { rvis[pix] = 0; continue; }
        uint32_t bits = rvis[pix];
        for (int i = 1; i <= good; ++i) bits |= (uint32_t)1u << (SMVS_CROSS_MAX_SRC - 1 - idx[i]);
        rvis[pix] = bits;
        const int nth = (int)((good - 1) * 0.5);
        bubble_sort(dd, good - 1); /* sorts entries [0, good - 1) of good (:3913) */
        out[pix] = dd[nth] / (thr * depth);
      }
  }
done:
  for (int v = 0; v < nv; ++v) free(zeros[v]);
  free(zeros);
  free(dmap);
  return st;
}

int orc_cross_filter_dedup_depth(const smvs_filter_view* view, const float* refined, const uint32_t* vis,
                                 float* out) {
  if (!view || !vis || !out) return SMVS_EINVAL;
  const size_t WH = (size_t)view->width * view->height;
  const float* d = view->ref_flag ? refined : view->depth;
  for (size_t k = 0; k < WH; ++k) out[k] = (d && (vis[k] & VIS_KEEP)) ? d[k] : 0.0f;
  return SMVS_OK;
}

int orc_cross_filter_poses(const smvs_filter_view* views, int num_views, const smvs_filter_problem* problem,
                           float refK[4], float refiK[4], float* poses) {
  if (check_set(views, num_views, problem, 1)) return SMVS_EINVAL;
  problem_poses(views, problem, refK, refiK, poses);
  return SMVS_OK;
}

int orc_encode_normal_map(const float* normal, int width, int height, uint32_t* code) {
  if (!normal || !code || width < 0 || height < 0) return SMVS_EINVAL;
  const size_t WH = (size_t)width * height;
  for (size_t k = 0; k < WH; ++k) code[k] = encode_normal(normal[k], normal[WH + k], normal[2 * WH + k]);
  return SMVS_OK;
}
