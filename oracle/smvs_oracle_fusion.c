/*
 * smvs_oracle_fusion.c — CPU oracle of the depth-map fusion.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of sensemap_b200/csrc/smvs_fusion.cu
 * and the CPU arm of its benchmark; the product never links or calls it.
 *
 * Restates StereoFusion (SenseMap src/mvs/fusion.cc) for one cluster holding
 * every image: the image loop of Run (:1160-1215) in FindNextImage order
 * (:697-727), FuseImage (:1730-1792) with its row slices taken one after
 * another, and Fuse (:1794-2182) — the depth-first traversal with its explicit
 * stack, the consistency tests against the seed pixel, and the medians of the
 * fused cluster. The reference's Eigen expressions are evaluated in the order
 * Eigen 3.3 uses for them with SSE and no FMA (the reference's flags, its
 * CMakeLists.txt:124-126):
 *   - a 3x4 matrix times a Vector4f is one packet product reduced as
 *     (p0 + p2) + (p1 + p3) (P_ * fused_ref_point :1895, inv_P_ * (...) :1954);
 *   - P_ * xyz.homogeneous() (:2081) is the 3x3 block product plus the last
 *     column, ((p0 + p1) + p2) + p3;
 *   - a 3x3 matrix times a Vector3f and dot products of Vector3f are
 *     ((p0 + p1) + p2).
 * Built with -ffp-contract=off so no multiply-add is fused. The CUDA unit
 * performs the same IEEE single-precision operations in the same order.
 * Differences from the reference, shared with the CUDA unit:
 *   - the inverse projection matrix is the float P inverted in double and
 *     rounded once (the reference inverts in float with Eigen's 4x4 routine);
 *   - a non-finite depth is skipped like a depth <= 0 (the reference converts
 *     the resulting NaN pixel coordinates to int, which is undefined);
 *   - a point's images are listed in ascending order (the reference uses the
 *     iteration order of a std::unordered_set).
 * Semantic maps, the ROI box, plane fitting and the clean-up passes after
 * fusion are not part of this path.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

#include "smvs_oracle.h"

#define BLANK 3 /* blank_size, fusion.cc:1757 and :1831 */

typedef struct {
  float P[12];     /* ComposeProjectionMatrix (src/mvs/utils.cc:35-42) */
  float iP[12];    /* ComposeInverseProjectionMatrix (:44-52), see header */
  float iR[9];     /* inv_R_ = R^T (:1047-1048) */
  int W, H;
} fview;

typedef struct {
  int view, row, col, depth;
} fentry;

typedef struct {
  size_t num_points, cap_points, num_vis, cap_vis;
  smvs_fused_point* points;
  uint64_t* vis_offsets; /* num_points + 1 */
  uint32_t* vis_images;
  int* order;
  int order_count;
  uint8_t** masks;
  int num_views;
} orc_fusion;

/* P = K [R | T] in float: Eigen's packet product of a 3x3 and a 3x4 row-major
 * matrix accumulates k = 0, 1, 2 in order. */
static void compose_P(const float K[9], const float R[9], const float T[3], float P[12]) {
  float M[12];
  for (int r = 0; r < 3; ++r) {
    M[4 * r] = R[3 * r];
    M[4 * r + 1] = R[3 * r + 1];
    M[4 * r + 2] = R[3 * r + 2];
    M[4 * r + 3] = T[r];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) P[4 * i + j] = (K[3 * i] * M[j] + K[3 * i + 1] * M[4 + j]) + K[3 * i + 2] * M[8 + j];
}

/* [P; 0 0 0 1]^-1, top three rows: [M^-1 | -M^-1 p] in double, rounded once. */
static void compose_inv_P(const float P[12], float iP[12]) {
  const double m0 = P[0], m1 = P[1], m2 = P[2], m3 = P[4], m4 = P[5], m5 = P[6], m6 = P[8], m7 = P[9], m8 = P[10];
  const double c00 = m4 * m8 - m5 * m7, c01 = m2 * m7 - m1 * m8, c02 = m1 * m5 - m2 * m4;
  const double c10 = m5 * m6 - m3 * m8, c11 = m0 * m8 - m2 * m6, c12 = m2 * m3 - m0 * m5;
  const double c20 = m3 * m7 - m4 * m6, c21 = m1 * m6 - m0 * m7, c22 = m0 * m4 - m1 * m3;
  const double det = m0 * c00 + m1 * c10 + m2 * c20;
  const double inv[9] = {c00 / det, c01 / det, c02 / det, c10 / det, c11 / det,
                         c12 / det, c20 / det, c21 / det, c22 / det};
  const double p[3] = {P[3], P[7], P[11]};
  for (int i = 0; i < 3; ++i) {
    iP[4 * i] = (float)inv[3 * i];
    iP[4 * i + 1] = (float)inv[3 * i + 1];
    iP[4 * i + 2] = (float)inv[3 * i + 2];
    iP[4 * i + 3] = (float)(-(inv[3 * i] * p[0] + inv[3 * i + 1] * p[1] + inv[3 * i + 2] * p[2]));
  }
}

/* Row i of a 3x4 matrix times (x, y, z, w): one SSE packet, predux. */
static inline float dot4p(const float* a, float x, float y, float z, float w) {
  return (a[0] * x + a[2] * z) + (a[1] * y + a[3] * w);
}
/* Row i of a 3x4 matrix times xyz.homogeneous(). */
static inline float dot3h(const float* a, float x, float y, float z) {
  return ((a[0] * x + a[1] * y) + a[2] * z) + a[3];
}

static int cmp_float(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}
static int cmp_u32(const void* a, const void* b) {
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

/* internal::Median (fusion.cc:47-60): the middle order statistic, or the mean
 * of the two middle ones for an even count. Sorts v in place. */
static float median(float* v, size_t n) {
  qsort(v, n, sizeof(float), cmp_float);
  const size_t mid = n / 2;
  if (n % 2 == 0) return (v[mid] + v[mid - 1]) / 2.0f;
  return v[mid];
}

/* StereoFusion::FindNextImage (fusion.cc:697-727). */
static int find_next_image(int prev, int nv, const int32_t* ov_off, const int32_t* ov_img, const uint8_t* used,
                           const uint8_t* fused, const smvs_fusion_view* views) {
  for (int pass = 0; pass < 2; ++pass)
    for (int32_t k = ov_off[prev]; k < ov_off[prev + 1]; ++k) {
      const int i = ov_img[k];
      if (used[i] && !fused[i] && (pass == 1 || !views[i].is_rig)) return i;
    }
  for (int pass = 0; pass < 2; ++pass)
    for (int i = 0; i < nv; ++i)
      if (used[i] && !fused[i] && (pass == 1 || !views[i].is_rig)) return i;
  return -1;
}

typedef struct {
  float *x, *y, *z, *nx, *ny, *nz, *c, *r, *g, *b, *err;
  uint32_t* vis;
  size_t cap;
} cluster;

static int cluster_reserve(cluster* cl, size_t n) {
  if (n <= cl->cap) return 0;
  size_t cap = cl->cap ? cl->cap * 2 : 256;
  while (cap < n) cap *= 2;
  float** f[] = {&cl->x, &cl->y, &cl->z, &cl->nx, &cl->ny, &cl->nz, &cl->c, &cl->r, &cl->g, &cl->b, &cl->err};
  for (size_t k = 0; k < sizeof(f) / sizeof(f[0]); ++k) {
    float* p = (float*)realloc(*f[k], cap * sizeof(float));
    if (!p) return -1;
    *f[k] = p;
  }
  uint32_t* v = (uint32_t*)realloc(cl->vis, cap * sizeof(uint32_t));
  if (!v) return -1;
  cl->vis = v;
  cl->cap = cap;
  return 0;
}

static void cluster_free(cluster* cl) {
  float* f[] = {cl->x, cl->y, cl->z, cl->nx, cl->ny, cl->nz, cl->c, cl->r, cl->g, cl->b, cl->err};
  for (size_t k = 0; k < sizeof(f) / sizeof(f[0]); ++k) free(f[k]);
  free(cl->vis);
}

typedef struct {
  const smvs_fusion_options* opt;
  const smvs_fusion_view* views;
  const fview* fv;
  int nv;
  const int32_t* ov_off;
  const int32_t* ov_img;
  const uint8_t* used;
  const uint8_t* fused;
  uint8_t** masks;
  float max_sq_reproj, min_cos_normal;
  fentry* stack;
  size_t stack_cap;
  cluster cl;
  orc_fusion* out;
} fuse_ctx;

static int push_entry(fuse_ctx* c, size_t* top, fentry e) {
  if (*top == c->stack_cap) {
    const size_t cap = c->stack_cap ? c->stack_cap * 2 : 1024;
    fentry* s = (fentry*)realloc(c->stack, cap * sizeof(fentry));
    if (!s) return -1;
    c->stack = s;
    c->stack_cap = cap;
  }
  c->stack[(*top)++] = e;
  return 0;
}

static int emit_point(fuse_ctx* c, const smvs_fused_point* p, const uint32_t* vis, size_t nvis) {
  orc_fusion* o = c->out;
  if (o->num_points == o->cap_points) {
    const size_t cap = o->cap_points ? o->cap_points * 2 : 4096;
    smvs_fused_point* np = (smvs_fused_point*)realloc(o->points, cap * sizeof(smvs_fused_point));
    uint64_t* no = (uint64_t*)realloc(o->vis_offsets, (cap + 1) * sizeof(uint64_t));
    if (np) o->points = np;
    if (no) o->vis_offsets = no;
    if (!np || !no) return -1;
    o->cap_points = cap;
  }
  if (o->num_vis + nvis > o->cap_vis) {
    size_t cap = o->cap_vis ? o->cap_vis * 2 : 16384;
    while (cap < o->num_vis + nvis) cap *= 2;
    uint32_t* nvp = (uint32_t*)realloc(o->vis_images, cap * sizeof(uint32_t));
    if (!nvp) return -1;
    o->vis_images = nvp;
    o->cap_vis = cap;
  }
  o->points[o->num_points] = *p;
  memcpy(o->vis_images + o->num_vis, vis, nvis * sizeof(uint32_t));
  o->num_vis += nvis;
  o->num_points++;
  o->vis_offsets[o->num_points] = o->num_vis;
  return 0;
}

/* StereoFusion::Fuse (fusion.cc:1794-2182) from one seed pixel. */
static int fuse(fuse_ctx* c, int image, int row0, int col0) {
  const smvs_fusion_options* opt = c->opt;
  cluster* cl = &c->cl;
  size_t n = 0, nerr = 0, top = 0;
  float ref[3] = {0, 0, 0}, ref_n[3] = {0, 0, 0};
  fentry e0 = {image, row0, col0, 0};
  if (push_entry(c, &top, e0)) return -1;
  while (top > 0) {
    const fentry e = c->stack[--top];
    const fview* v = &c->fv[e.view];
    const size_t pix = (size_t)e.row * v->W + e.col;
    uint8_t* mask = c->masks[e.view];
    if (__atomic_load_n(&mask[pix], __ATOMIC_RELAXED)) continue;
    const float depth = c->views[e.view].depth[pix];
    if (!(depth > 0.0f) || !isfinite(depth)) continue;
    float depth_error = 0.0f;
    if (e.depth > 0) {
      const float p0 = dot4p(v->P, ref[0], ref[1], ref[2], 1.0f);
      const float p1 = dot4p(v->P + 4, ref[0], ref[1], ref[2], 1.0f);
      const float p2 = dot4p(v->P + 8, ref[0], ref[1], ref[2], 1.0f);
      const float col_diff = p0 / p2 - (float)e.col;
      const float row_diff = p1 / p2 - (float)e.row;
      const float sq = col_diff * col_diff + row_diff * row_diff;
      if (sq > c->max_sq_reproj) continue;
      depth_error = fabsf(p2 - depth) / depth;
      if ((double)depth_error > opt->max_depth_error) continue;
    }
    float nrm[3] = {0, 0, 0};
    if (opt->with_normal) {
      const float* nm = c->views[e.view].normal;
      const size_t plane = (size_t)v->W * v->H;
      const float n0 = nm[pix], n1 = nm[plane + pix], n2 = nm[2 * plane + pix];
      for (int i = 0; i < 3; ++i) nrm[i] = (v->iR[3 * i] * n0 + v->iR[3 * i + 1] * n1) + v->iR[3 * i + 2] * n2;
      if (e.depth > 0) {
        const float cos_err = (ref_n[0] * nrm[0] + ref_n[1] * nrm[1]) + ref_n[2] * nrm[2];
        if (cos_err < c->min_cos_normal) continue;
      }
    }
    const float cd = (float)e.col * depth, rd = (float)e.row * depth;
    const float xyz[3] = {dot4p(v->iP, cd, rd, depth, 1.0f), dot4p(v->iP + 4, cd, rd, depth, 1.0f),
                          dot4p(v->iP + 8, cd, rd, depth, 1.0f)};
    /* Color of the pixel and the red-channel gradient (:2005-2021). */
    const uint8_t* img = c->views[e.view].color;
    uint8_t rgb[3] = {0, 0, 0};
    float grad = 0.0f;
    if (img) {
      const uint8_t* px = img + 3 * pix;
      rgb[0] = px[0];
      rgb[1] = px[1];
      rgb[2] = px[2];
      if (e.col > 1 && e.col < v->W - 1 && e.row > 1 && e.row < v->H - 1) {
        const float gx = (float)((int)img[3 * (pix - 1)] - (int)img[3 * (pix + 1)]) / 255.0f;
        const float gy = (float)((int)img[3 * (pix - v->W)] - (int)img[3 * (pix + v->W)]) / 255.0f;
        grad = sqrtf(gx * gx + gy * gy);
      }
    }
    __atomic_store_n(&mask[pix], (uint8_t)1, __ATOMIC_RELAXED);
    if (cluster_reserve(cl, n + 1)) return -1;
    cl->x[n] = xyz[0];
    cl->y[n] = xyz[1];
    cl->z[n] = xyz[2];
    cl->nx[n] = nrm[0];
    cl->ny[n] = nrm[1];
    cl->nz[n] = nrm[2];
    cl->c[n] = grad;
    cl->r[n] = rgb[0];
    cl->g[n] = rgb[1];
    cl->b[n] = rgb[2];
    cl->vis[n] = (uint32_t)e.view;
    if (e.depth > 0) cl->err[nerr++] = depth_error;
    ++n;
    if (e.depth == 0) {
      ref[0] = xyz[0];
      ref[1] = xyz[1];
      ref[2] = xyz[2];
      ref_n[0] = nrm[0];
      ref_n[1] = nrm[1];
      ref_n[2] = nrm[2];
    }
    if (n >= (size_t)opt->max_num_pixels) break;
    if (e.depth + 1 >= opt->max_traversal_depth) continue;
    for (int32_t k = c->ov_off[e.view]; k < c->ov_off[e.view + 1]; ++k) {
      const int u = c->ov_img[k];
      if (!c->used[u] || c->fused[u]) continue;
      const fview* fu = &c->fv[u];
      const float q0 = dot3h(fu->P, xyz[0], xyz[1], xyz[2]);
      const float q1 = dot3h(fu->P + 4, xyz[0], xyz[1], xyz[2]);
      const float q2 = dot3h(fu->P + 8, xyz[0], xyz[1], xyz[2]);
      const float ucol = roundf(q0 / q2), urow = roundf(q1 / q2);
      if (!(ucol >= (float)BLANK && urow >= (float)BLANK && ucol < (float)(fu->W - BLANK) &&
            urow < (float)(fu->H - BLANK)))
        continue;
      fentry ne = {u, (int)urow, (int)ucol, e.depth + 1};
      if (push_entry(c, &top, ne)) return -1;
    }
  }
  /* The fused point (:2098-2180). */
  if (n < (size_t)opt->min_num_pixels) return 0;
  qsort(cl->vis, n, sizeof(uint32_t), cmp_u32);
  size_t nvis = 0;
  for (size_t i = 0; i < n; ++i)
    if (i == 0 || cl->vis[i] != cl->vis[i - 1]) cl->vis[nvis++] = cl->vis[i];
  if (nvis < (size_t)opt->min_num_visible_images) return 0;
  smvs_fused_point p;
  memset(&p, 0, sizeof(p));
  p.x = median(cl->x, n);
  p.y = median(cl->y, n);
  p.z = median(cl->z, n);
  if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) return 0;
  if (opt->with_normal) {
    const float fx = median(cl->nx, n), fy = median(cl->ny, n), fz = median(cl->nz, n);
    const float norm = sqrtf((fx * fx + fy * fy) + fz * fz);
    if (norm < FLT_EPSILON) return 0;
    p.nx = fx / norm;
    p.ny = fy / norm;
    p.nz = fz / norm;
  }
  const float* chan[3] = {cl->r, cl->g, cl->b};
  uint8_t rgb[3];
  for (int k = 0; k < 3; ++k) {
    float m = roundf(median((float*)chan[k], n));
    m = m < 255.0f ? m : 255.0f; /* TruncateCast<float, uint8_t> (src/util/math.h:341-345) */
    m = m > 0.0f ? m : 0.0f;
    rgb[k] = (uint8_t)m;
  }
  p.r = rgb[0];
  p.g = rgb[1];
  p.b = rgb[2];
  float m_conf = 0.0f;
  for (size_t i = 0; i < n; ++i) m_conf += cl->c[i];
  m_conf /= (float)n;
  if (nvis >= 3) m_conf = 1.0f;
  m_conf = 1.0f - m_conf;
  float score = (float)((double)median(cl->err, nerr) / opt->max_depth_error);
  const float mixed = 0.6f * score + 0.4f * m_conf;
  score = (1.0f < mixed) ? 1.0f : mixed;
  if (!isfinite(score)) return 0;
  p.score = score;
  int rc;
#pragma omp critical(orc_fusion_emit)
  rc = emit_point(c, &p, cl->vis, nvis);
  return rc;
}

void* orc_fusion_run(const smvs_fusion_options* opt, const smvs_fusion_view* views, int nv, const int32_t* ov_off,
                     const int32_t* ov_img, int max_images) {
  return orc_fusion_run_threads(opt, views, nv, ov_off, ov_img, max_images, 1);
}

/* threads > 1: the reference's concurrent FuseImage (:1201-1205): `threads`
 * row slices of each image run at once on that many OpenMP threads, sharing
 * the pixel masks without order (relaxed atomics where the reference races)
 * and appending points under a lock. Results then depend on the timing, as
 * the reference's do: this form is a timing baseline, not a checker. */
void* orc_fusion_run_threads(const smvs_fusion_options* opt, const smvs_fusion_view* views, int nv,
                             const int32_t* ov_off, const int32_t* ov_img, int max_images, int threads) {
  if (!opt || !views || nv < 1 || !ov_off || (ov_off[nv] > 0 && !ov_img) || opt->min_num_pixels < 2 ||
      opt->max_num_pixels < opt->min_num_pixels || opt->max_traversal_depth < 1 || opt->step_size < 1 ||
      opt->num_slices < 1 || opt->min_num_visible_images < 0)
    return NULL;
  for (int v = 0; v < nv; ++v) {
    if (views[v].depth && (views[v].width < 1 || views[v].height < 1 || (opt->with_normal && !views[v].normal)))
      return NULL;
    for (int32_t k = ov_off[v]; k < ov_off[v + 1]; ++k)
      if (ov_img[k] < 0 || ov_img[k] >= nv) return NULL;
  }
  orc_fusion* o = (orc_fusion*)calloc(1, sizeof(orc_fusion));
  fview* fv = (fview*)calloc((size_t)nv, sizeof(fview));
  uint8_t* used = (uint8_t*)calloc((size_t)nv, 1);
  uint8_t* fused = (uint8_t*)calloc((size_t)nv, 1);
  o->masks = (uint8_t**)calloc((size_t)nv, sizeof(uint8_t*));
  o->order = (int*)calloc((size_t)nv, sizeof(int));
  o->vis_offsets = (uint64_t*)calloc(1, sizeof(uint64_t));
  o->num_views = nv;
  fuse_ctx c;
  memset(&c, 0, sizeof(c));
  int ok = o && fv && used && fused && o->masks && o->order && o->vis_offsets;
  for (int v = 0; ok && v < nv; ++v) {
    fv[v].W = views[v].width;
    fv[v].H = views[v].height;
    compose_P(views[v].K, views[v].R, views[v].T, fv[v].P);
    compose_inv_P(fv[v].P, fv[v].iP);
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) fv[v].iR[3 * i + k] = views[v].R[3 * k + i];
    used[v] = views[v].depth != NULL;
    if (used[v]) {
      o->masks[v] = (uint8_t*)calloc((size_t)views[v].width * views[v].height, 1);
      ok = o->masks[v] != NULL;
    }
  }
  if (ok) {
    c.opt = opt;
    c.views = views;
    c.fv = fv;
    c.nv = nv;
    c.ov_off = ov_off;
    c.ov_img = ov_img;
    c.used = used;
    c.fused = fused;
    c.masks = o->masks;
    c.out = o;
    c.max_sq_reproj = (float)(opt->max_reproj_error * opt->max_reproj_error);
    c.min_cos_normal =
        (float)cos(opt->max_normal_error * 0.0174532925199432954743716805978692718781530857086181640625);
    /* Run's image loop (:1151-1215). */
    int start = 0;
    for (int i = 0; i < nv; ++i)
      if (!views[i].is_rig) {
        start = i;
        break;
      }
    for (int image = start; ok && image >= 0; image = find_next_image(image, nv, ov_off, ov_img, used, fused, views)) {
      if (!used[image]) continue;
      if (max_images > 0 && o->order_count >= max_images) break;
      const int W = views[image].width, H = views[image].height;
      const int T = threads > 1 ? threads : opt->num_slices;
      const int hs = (H + T - 1) / T;
      if (threads <= 1) {
        for (int t = 0; ok && t < T; ++t) { /* FuseImage (:1730-1792), slice t */
          const int limit = hs * (t + 1) < H ? hs * (t + 1) : H;
          const int row_end = limit < H - BLANK ? limit : H - BLANK;
          for (int row = hs * t > BLANK ? hs * t : BLANK; ok && row < row_end; row += opt->step_size)
            for (int col = BLANK; ok && col < W - BLANK; col += opt->step_size) {
              if (o->masks[image][(size_t)row * W + col]) continue;
              ok = fuse(&c, image, row, col) == 0;
            }
        }
      } else {
        int failed = 0;
#pragma omp parallel num_threads(T)
        {
          fuse_ctx lc = c;
          lc.stack = NULL;
          lc.stack_cap = 0;
          memset(&lc.cl, 0, sizeof(lc.cl));
          for (int t = omp_get_thread_num(); t < T; t += omp_get_num_threads()) {
            const int limit = hs * (t + 1) < H ? hs * (t + 1) : H;
            const int row_end = limit < H - BLANK ? limit : H - BLANK;
            for (int row = hs * t > BLANK ? hs * t : BLANK; row < row_end; row += opt->step_size)
              for (int col = BLANK; col < W - BLANK; col += opt->step_size) {
                if (__atomic_load_n(&o->masks[image][(size_t)row * W + col], __ATOMIC_RELAXED)) continue;
                if (fuse(&lc, image, row, col)) __atomic_store_n(&failed, 1, __ATOMIC_RELAXED);
              }
          }
          cluster_free(&lc.cl);
          free(lc.stack);
        }
        ok = !failed;
      }
      fused[image] = 255;
      o->order[o->order_count++] = image;
    }
  }
  cluster_free(&c.cl);
  free(c.stack);
  free(fv);
  free(used);
  free(fused);
  if (!ok) {
    orc_fusion_free(o);
    return NULL;
  }
  return o;
}

int orc_fusion_sizes(void* h, size_t* num_points, size_t* num_vis, int* order_count) {
  orc_fusion* o = (orc_fusion*)h;
  if (!o) return SMVS_EINVAL;
  if (num_points) *num_points = o->num_points;
  if (num_vis) *num_vis = o->num_vis;
  if (order_count) *order_count = o->order_count;
  return SMVS_OK;
}

int orc_fusion_copy(void* h, smvs_fused_point* points, uint64_t* vis_offsets, uint32_t* vis_images, int* order) {
  orc_fusion* o = (orc_fusion*)h;
  if (!o) return SMVS_EINVAL;
  if (points && o->num_points) memcpy(points, o->points, o->num_points * sizeof(smvs_fused_point));
  if (vis_offsets) memcpy(vis_offsets, o->vis_offsets, (o->num_points + 1) * sizeof(uint64_t));
  if (vis_images && o->num_vis) memcpy(vis_images, o->vis_images, o->num_vis * sizeof(uint32_t));
  if (order && o->order_count) memcpy(order, o->order, (size_t)o->order_count * sizeof(int));
  return SMVS_OK;
}

/* The view's fused-pixel mask (all zero for an unused view). */
int orc_fusion_mask(void* h, int view, int width, int height, uint8_t* out) {
  orc_fusion* o = (orc_fusion*)h;
  if (!o || view < 0 || view >= o->num_views || !out) return SMVS_EINVAL;
  if (o->masks[view])
    memcpy(out, o->masks[view], (size_t)width * height);
  else
    memset(out, 0, (size_t)width * height);
  return SMVS_OK;
}

void orc_fusion_free(void* h) {
  orc_fusion* o = (orc_fusion*)h;
  if (!o) return;
  if (o->masks)
    for (int v = 0; v < o->num_views; ++v) free(o->masks[v]);
  free(o->masks);
  free(o->points);
  free(o->vis_offsets);
  free(o->vis_images);
  free(o->order);
  free(o);
}

/* ------------------------------------------------------------------------ */
/* Clean-up passes after the image loop, over a fused cloud given as arrays.  */
/* ------------------------------------------------------------------------ */

/* RemoveDuplicatePoints, fusion.cc:2184-2266: keep[i] = 0 for the points it
 * drops. The projection is Eigen's float K * (R * X + T) (3x3 products reduce
 * as (p0 + p1) + p2) and std::round of proj / z; a point's images are visited
 * in the order given (ascending in this library). */
int orc_fusion_duplicate_keep(const smvs_fusion_view* views, int nv, const smvs_fused_point* pts, size_t n,
                              const uint64_t* off, const uint32_t* vis, uint8_t* keep) {
  if (!views || nv < 1 || (n && (!pts || !off || !vis)) || !keep) return SMVS_EINVAL;
  int64_t** occ = (int64_t**)calloc((size_t)nv, sizeof(int64_t*));
  uint8_t* removal = (uint8_t*)calloc(n ? n : 1, 1);
  if (!occ || !removal) { free(occ); free(removal); return SMVS_ENOMEM; }
  for (int v = 0; v < nv; ++v) {
    const size_t plane = (size_t)views[v].width * views[v].height;
    occ[v] = (int64_t*)malloc(sizeof(int64_t) * (plane ? plane : 1));
    if (!occ[v]) {
      for (int k = 0; k < v; ++k) free(occ[k]);
      free(occ); free(removal);
      return SMVS_ENOMEM;
    }
    for (size_t q = 0; q < plane; ++q) occ[v][q] = -1;
  }
  for (size_t i = 0; i < n; ++i) {
    if (removal[i]) continue;
    const uint64_t nvis = off[i + 1] - off[i];
    const float X[3] = {pts[i].x, pts[i].y, pts[i].z};
    for (uint64_t k = off[i]; k < off[i + 1]; ++k) {
      const int img = (int)vis[k];
      if (img < 0 || img >= nv) continue;
      const smvs_fusion_view* v = &views[img];
      float c[3], q[3];
      for (int r = 0; r < 3; ++r) c[r] = ((v->R[3 * r] * X[0] + v->R[3 * r + 1] * X[1]) + v->R[3 * r + 2] * X[2]) + v->T[r];
      for (int r = 0; r < 3; ++r) q[r] = (v->K[3 * r] * c[0] + v->K[3 * r + 1] * c[1]) + v->K[3 * r + 2] * c[2];
      const int u = (int)roundf(q[0] / q[2]);
      const int w = (int)roundf(q[1] / q[2]);
      if (u < 0 || u >= v->width || w < 0 || w >= v->height) continue;
      int64_t* o = &occ[img][(size_t)w * v->width + u];
      if (*o == -1) { *o = (int64_t)i; continue; }
      if (off[*o + 1] - off[*o] > nvis) { removal[i] = 1; break; }
      removal[*o] = 1;
      *o = (int64_t)i;
    }
  }
  for (size_t i = 0; i < n; ++i) keep[i] = !removal[i];
  for (int v = 0; v < nv; ++v) free(occ[v]);
  free(occ);
  free(removal);
  return SMVS_OK;
}

/* ComputeAverageDistance (patch_match_controller.cc:115-228) by brute force:
 * each point's K = nb + 1 nearest points (itself included) by squared distance
 * in double (dx^2 + dy^2 + dz^2 summed in that order, CGAL's Euclidean
 * distance), their square roots added nearest first into a float, over K - 1.
 * Then RemoveOutliers (fusion.cc:2542-2611). scores (n) are updated in place;
 * spacing (n, may be NULL) receives the per-point spacings. */
int orc_fusion_outlier_keep(const smvs_fused_point* pts, size_t n, int nb, double max_spacing_factor, float* scores,
                            uint8_t* keep, float* spacing) {
  if ((n && (!pts || !scores || !keep)) || nb < 1 || nb > 63 || !(max_spacing_factor > 0)) return SMVS_EINVAL;
  if (n == 0) return SMVS_OK;
  const int K = nb + 1;
  float* sp = (float*)malloc(sizeof(float) * n);
  if (!sp) return SMVS_ENOMEM;
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t i = 0; i < n; ++i) {
    double best[64];
    int cnt = 0;
    const double qx = pts[i].x, qy = pts[i].y, qz = pts[i].z;
    for (size_t j = 0; j < n; ++j) {
      const double dx = qx - (double)pts[j].x, dy = qy - (double)pts[j].y, dz = qz - (double)pts[j].z;
      double d = dx * dx;
      d += dy * dy;
      d += dz * dz;
      if (cnt < K) {
        int m = cnt++;
        while (m > 0 && best[m - 1] > d) { best[m] = best[m - 1]; --m; }
        best[m] = d;
      } else if (d < best[K - 1]) {
        int m = K - 1;
        while (m > 0 && best[m - 1] > d) { best[m] = best[m - 1]; --m; }
        best[m] = d;
      }
    }
    float s = 0.0f;
    for (int k = 0; k < cnt; ++k) s = (float)((double)s + sqrt(best[k]));
    if (cnt > 1) s /= (float)(cnt - 1);
    sp[i] = s;
  }
  float average = 0.0f;
  for (size_t i = 0; i < n; ++i) average += sp[i];
  average /= (float)n;
  if (average > 1e-6) {
    for (size_t i = 0; i < n; ++i) {
      const float factor = (float)((double)sp[i] / (max_spacing_factor * (double)average));
      scores[i] = (float)((double)scores[i] * 0.6 + (double)factor * 0.4);
    }
  }
  float smin = scores[0], smax = scores[0];
  for (size_t i = 0; i < n; ++i) {
    if (scores[i] < smin) smin = scores[i];
    if (scores[i] > smax) smax = scores[i];
  }
  const float range = smax - smin;
  float ratios[256] = {0}, acc[256];
  for (size_t i = 0; i < n; ++i) {
    const int b = range > 0 ? (int)(((scores[i] - smin) / range) * 255) : 0;
    ratios[b]++;
  }
  for (int k = 0; k < 256; ++k) ratios[k] /= (float)n;
  float sum = 0.0f;
  for (int k = 0; k < 256; ++k) { sum += ratios[k]; acc[k] = sum; }
  for (size_t i = 0; i < n; ++i) {
    const int b = range > 0 ? (int)(((scores[i] - smin) / range) * 255) : 0;
    keep[i] = !((double)ratios[b] < 0.01 && (double)acc[b] >= 0.9);
  }
  if (spacing) memcpy(spacing, sp, sizeof(float) * n);
  free(sp);
  return SMVS_OK;
}
