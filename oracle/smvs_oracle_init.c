/*
 * smvs_oracle_init.c — CPU oracle of the depth initialisation from a model.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of sensemap_b200/csrc/smvs_init_maps.cu;
 * the product never links or calls it.
 *
 * Restates, sequentially and in the reference's loop order, the initial
 * depth/normal maps PatchMatchController builds before a PatchMatch pass
 * (SenseMap src/controllers/patch_match_controller.cc):
 *   - InitDepthMap (:1205-1307) projecting the sparse points that the view
 *     observes, then InitDepthMapFromSparsePoint (:483-518) splatting them
 *     into 7x7 windows with a depth test;
 *   - Model2Depth (:520-642) rasterising a triangle mesh with a depth test;
 *   - Ply2Depth (:643-750) splatting oriented dense points.
 * The reference evaluates the sparse path in float and the mesh and dense-point
 * paths in double through Eigen; this file writes every sum, product and
 * division in a fixed order (built with -ffp-contract=off), which the CUDA unit
 * repeats exactly. The sequential depth tests here (first writer wins ties,
 * later writers win only below the stored float) are what the CUDA unit's
 * order-independent passes must reproduce.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "smvs_oracle.h"

/* x = M y + t, row-major 3x3, float, left-to-right sums. */
static void mat3_apply_f(const float* M, const float* y, const float* t, float* x) {
  for (int r = 0; r < 3; ++r) {
    float s = M[3 * r] * y[0] + M[3 * r + 1] * y[1] + M[3 * r + 2] * y[2];
    x[r] = t ? s + t[r] : s;
  }
}

static void mat3_apply_d(const double* M, const double* y, const double* t, double* x) {
  for (int r = 0; r < 3; ++r) {
    double s = M[3 * r] * y[0] + M[3 * r + 1] * y[1] + M[3 * r + 2] * y[2];
    x[r] = t ? s + t[r] : s;
  }
}

static double dot3d(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* double -> int truncation for pixel bounds; values beyond +-2^30 (where the
 * reference's conversion is undefined) are clamped, NaN gives -2^30. */
static int to_int(double x) {
  if (x != x) return -1073741824;
  return (int)fmin(fmax(x, -1073741824.0), 1073741824.0);
}

/* 3x3 inverse by the adjugate (the closed form Eigen uses for 3x3 matrices). */
static void inverse3d(const double* m, double* inv) {
  const double c00 = m[4] * m[8] - m[5] * m[7];
  const double c01 = m[5] * m[6] - m[3] * m[8];
  const double c02 = m[3] * m[7] - m[4] * m[6];
  const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  const double id = 1.0 / det;
  inv[0] = c00 * id;
  inv[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  inv[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  inv[3] = c01 * id;
  inv[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  inv[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  inv[6] = c02 * id;
  inv[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  inv[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

static void finish_range(float lo, float hi, float* range) {
  if (lo == FLT_MAX) { lo = 0.0f; hi = 100.0f; } /* :1297-1300 */
  range[0] = 0.000001f;                          /* first *= 0.9 is overwritten (:1301-1304) */
  range[1] = hi * 1.1f;
}

int orc_init_from_sparse_points(const smvs_view* v, const float* xyz, size_t n, float* depth, float* normal,
                                float* range) {
  if (!v || (n && !xyz) || !depth || !normal || !range) return SMVS_EINVAL;
  const int W = v->width, H = v->height;
  memset(depth, 0, sizeof(float) * (size_t)W * H);
  memset(normal, 0, sizeof(float) * 3 * (size_t)W * H);
  float lo = FLT_MAX, hi = FLT_EPSILON;
  for (size_t i = 0; i < n; ++i) {
    /* Xc = K (R X + T) (:1241-1251) */
    float Y[3], Xc[3];
    mat3_apply_f(v->R, xyz + 3 * i, v->T, Y);
    mat3_apply_f(v->K, Y, NULL, Xc);
    if (!(Xc[2] > 0)) continue;
    /* int fu = Xc[0] / Xc[2] truncates toward zero, then 0 <= fu < W: the same
     * as -1 < Xc[0] / Xc[2] < W for finite values (and rejects the rest) */
    const float qu = Xc[0] / Xc[2], qv = Xc[1] / Xc[2];
    if (!(qu > -1.0f && qu < (float)W && qv > -1.0f && qv < (float)H)) continue;
    const int fu = (int)qu, fv = (int)qv;
    lo = fminf(lo, Xc[2]);
    hi = fmaxf(hi, Xc[2]);
    /* InitDepthMapFromSparsePoint (:494-517): 7x7 window, first writer keeps ties */
    const float z = Xc[2];
    const int u0 = fu - 3 > 0 ? fu - 3 : 0, u1 = fu + 3 < W - 1 ? fu + 3 : W - 1;
    const int v0 = fv - 3 > 0 ? fv - 3 : 0, v1 = fv + 3 < H - 1 ? fv + 3 : H - 1;
    for (int y = v0; y <= v1; ++y)
      for (int x = u0; x <= u1; ++x) {
        const float d = depth[(size_t)y * W + x];
        if (d == 0 || d > z) depth[(size_t)y * W + x] = z; /* normal stays (0, 0, 0) */
      }
  }
  finish_range(lo, hi, range);
  return SMVS_OK;
}

/* Camera-frame data shared by the double-precision paths. */
typedef struct {
  double K[9], R[9], T[3], Kinv[9], C[3], ray[3];
} cam_d;

static void cam_setup(const smvs_view* v, cam_d* c) {
  for (int k = 0; k < 9; ++k) { c->K[k] = v->K[k]; c->R[k] = v->R[k]; }
  for (int k = 0; k < 3; ++k) c->T[k] = v->T[k];
  inverse3d(c->K, c->Kinv);
  for (int r = 0; r < 3; ++r) c->C[r] = -(c->R[r] * c->T[0] + c->R[3 + r] * c->T[1] + c->R[6 + r] * c->T[2]);
  for (int k = 0; k < 3; ++k) c->ray[k] = c->R[6 + k];
}

/* Depth test of Model2Depth / Ply2Depth: nd == 0 || z < nd, z double. */
static void write_depth(float* depth, float* normal, size_t WH, size_t p, double z, const double* n, float* lo,
                        float* hi) {
  if (isnan(z)) return; /* not written (the reference stores a NaN when it is a pixel's first write) */
  const float nd = depth[p];
  if (nd == 0 || z < (double)nd) {
    depth[p] = (float)z;
    normal[p] = (float)n[0];
    normal[WH + p] = (float)n[1];
    normal[2 * WH + p] = (float)n[2];
    *lo = fminf(*lo, (float)z);
    *hi = fmaxf(*hi, (float)z);
  }
}

int orc_init_from_mesh(const smvs_view* v, const double* vert, size_t nvert, const int32_t* faces, size_t nface,
                       const double* face_normals, float* depth, float* normal, float* range) {
  if (!v || (nface && (!vert || !faces || !face_normals)) || !depth || !normal || !range) return SMVS_EINVAL;
  const int W = v->width, H = v->height;
  const size_t WH = (size_t)W * H;
  memset(depth, 0, sizeof(float) * WH);
  memset(normal, 0, sizeof(float) * 3 * WH);
  cam_d c;
  cam_setup(v, &c);
  const double thresh_fov = cos(90.0); /* [quirk] :536, 90 radians */
  float lo = FLT_MAX, hi = FLT_EPSILON;
  for (size_t f = 0; f < nface; ++f) {
    const int32_t* fa = faces + 3 * f;
    if (fa[0] < 0 || fa[1] < 0 || fa[2] < 0 || (size_t)fa[0] >= nvert || (size_t)fa[1] >= nvert ||
        (size_t)fa[2] >= nvert)
      return SMVS_EINVAL;
    const double* p[3] = {vert + 3 * (size_t)fa[0], vert + 3 * (size_t)fa[1], vert + 3 * (size_t)fa[2]};
    double cen[3], cc[3];
    for (int k = 0; k < 3; ++k) cen[k] = (p[0][k] + p[1][k] + p[2][k]) / 3;
    for (int k = 0; k < 3; ++k) cc[k] = cen[k] - c.C[k];
    if (dot3d(cc, face_normals + 3 * f) > 0) continue; /* back face (:557-559) */
    const double len = sqrt(dot3d(cc, cc));
    if (len > 0) for (int k = 0; k < 3; ++k) cc[k] = cc[k] / len; /* normalized() */
    if (dot3d(c.ray, cc) < thresh_fov) continue;
    double Xc[3][3], uv[3][3];
    for (int k = 0; k < 3; ++k) {
      mat3_apply_d(c.R, p[k], c.T, Xc[k]);
      mat3_apply_d(c.K, Xc[k], NULL, uv[k]);
      const double w = uv[k][2];
      uv[k][0] = uv[k][0] / w; uv[k][1] = uv[k][1] / w; uv[k][2] = uv[k][2] / w;
    }
    int u_min = to_int(fmin(uv[0][0], fmin(uv[1][0], uv[2][0])));
    int u_max = to_int(fmax(uv[0][0], fmax(uv[1][0], uv[2][0])));
    int v_min = to_int(fmin(uv[0][1], fmin(uv[1][1], uv[2][1])));
    int v_max = to_int(fmax(uv[0][1], fmax(uv[1][1], uv[2][1])));
    u_min = u_min > 0 ? u_min : 0;
    v_min = v_min > 0 ? v_min : 0;
    u_max = u_max < W - 1 ? u_max : W - 1;
    v_max = v_max < H - 1 ? v_max : H - 1;
    if (Xc[0][2] <= 0 || Xc[1][2] <= 0 || Xc[2][2] <= 0 || u_min > u_max || v_min > v_max) continue;
    double e1[3], e2[3], nn[3], np[3];
    for (int k = 0; k < 3; ++k) { e1[k] = Xc[1][k] - Xc[0][k]; e2[k] = Xc[2][k] - Xc[0][k]; }
    nn[0] = e1[1] * e2[2] - e1[2] * e2[1];
    nn[1] = e1[2] * e2[0] - e1[0] * e2[2];
    nn[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double nl = sqrt(dot3d(nn, nn));
    if (nl > 0) for (int k = 0; k < 3; ++k) nn[k] = nn[k] / nl;
    const double ip = 1.0 / dot3d(nn, Xc[0]);
    for (int k = 0; k < 3; ++k) np[k] = nn[k] * ip;
    const double a1x = uv[1][0] - uv[0][0], a1y = uv[1][1] - uv[0][1];
    const double a2x = uv[2][0] - uv[1][0], a2y = uv[2][1] - uv[1][1];
    const double a3x = uv[0][0] - uv[2][0], a3y = uv[0][1] - uv[2][1];
    for (int y = v_min; y <= v_max; ++y)
      for (int x = u_min; x <= u_max; ++x) {
        const double m1 = a1x * (y - uv[0][1]) - (x - uv[0][0]) * a1y;
        const double m2 = a2x * (y - uv[1][1]) - (x - uv[1][0]) * a2y;
        const double m3 = a3x * (y - uv[2][1]) - (x - uv[2][0]) * a3y;
        if (m1 < 0 && m2 < 0 && m3 < 0) {
          const double pix[3] = {(double)x, (double)y, 1.0};
          double xc[3];
          mat3_apply_d(c.Kinv, pix, NULL, xc);
          const double z = 1.0 / dot3d(np, xc);
          write_depth(depth, normal, WH, (size_t)y * W + x, z, nn, &lo, &hi);
        }
      }
  }
  finish_range(lo, hi, range);
  return SMVS_OK;
}

int orc_init_from_dense_points(const smvs_view* v, const float* xyz, const float* nrm, size_t n, int level,
                               float* depth, float* normal, float* range) {
  if (!v || (n && (!xyz || !nrm)) || !depth || !normal || !range || level < 0 || level > 8) return SMVS_EINVAL;
  const int W = v->width, H = v->height;
  const size_t WH = (size_t)W * H;
  memset(depth, 0, sizeof(float) * WH);
  memset(normal, 0, sizeof(float) * 3 * WH);
  cam_d c;
  cam_setup(v, &c);
  const int ws = 1 << level; /* std::pow(2, PLY_INIT_DEPTH_LEVEL) (:703) */
  float lo = FLT_MAX, hi = FLT_EPSILON;
  for (size_t i = 0; i < n; ++i) {
    const double cen[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    const double nw[3] = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
    double inrm[3], cc[3], Xc[3], uv[3];
    mat3_apply_d(c.R, nw, NULL, inrm);
    for (int k = 0; k < 3; ++k) cc[k] = cen[k] - c.C[k];
    if (dot3d(cc, nw) > 0) continue; /* :672-674 */
    mat3_apply_d(c.R, cen, c.T, Xc);
    mat3_apply_d(c.K, Xc, NULL, uv);
    uv[0] = uv[0] / uv[2];
    uv[1] = uv[1] / uv[2];
    if (Xc[2] <= 0 || !(uv[0] >= 0 && uv[1] >= 0 && uv[0] <= W - 1 && uv[1] <= H - 1)) continue; /* NaN too */
    const int i0 = (int)floor(uv[0]) - ws, i1 = (int)ceil(uv[0]) + ws;
    const int j0 = (int)floor(uv[1]) - ws, j1 = (int)ceil(uv[1]) + ws;
    for (int x = i0; x <= i1; ++x)
      for (int y = j0; y <= j1; ++y) {
        if (x < 0 || x > W - 1 || y < 0 || y > H - 1) continue;
        if (x % 2 == 0 || y % 2 == 0) continue; /* odd pixels only (:707-709) */
        write_depth(depth, normal, WH, (size_t)y * W + x, Xc[2], inrm, &lo, &hi);
      }
  }
  finish_range(lo, hi, range);
  return SMVS_OK;
}

/* ------------------------------------------------------------------------ */
/* Delaunay initial map: InitDepthMap's projection (:1236-1256) and           */
/* InitDepthMapFromDelaunay (:398-474) over a given triangulation.            */
/* ------------------------------------------------------------------------ */

/* The points that land in the view, in input order: their truncated pixel
 * positions uv[2k], uv[2k + 1], camera depths z[k] and input indices idx[k]. */
int orc_delaunay_points(const smvs_view* v, const float* xyz, size_t n, int32_t* uv, float* z, int32_t* idx,
                        size_t* count) {
  if (!v || (n && !xyz) || !uv || !z || !idx || !count) return SMVS_EINVAL;
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) {
    float Y[3], Xc[3];
    mat3_apply_f(v->R, xyz + 3 * i, v->T, Y);
    mat3_apply_f(v->K, Y, NULL, Xc);
    if (!(Xc[2] > 0)) continue;
    const float qu = Xc[0] / Xc[2], qv = Xc[1] / Xc[2];
    if (!(qu > -1.0f && qu < (float)v->width && qv > -1.0f && qv < (float)v->height)) continue;
    uv[2 * m] = (int)qu;
    uv[2 * m + 1] = (int)qv;
    z[m] = Xc[2];
    idx[m] = (int32_t)i;
    ++m;
  }
  *count = m;
  return SMVS_OK;
}

static float dot3f(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

/* tris: counter-clockwise triples of indices into the orc_delaunay_points
 * list. A pixel inside several triangles (on a shared edge) takes the one
 * whose vertex indices, sorted, are largest. */
int orc_init_from_delaunay(const smvs_view* v, const float* xyz, size_t n, const int32_t* tris, size_t ntri,
                           float* depth, float* normal, float* range) {
  if (!v || (n && !xyz) || (ntri && !tris) || !depth || !normal || !range) return SMVS_EINVAL;
  const int W = v->width, H = v->height;
  const size_t WH = (size_t)W * H;
  int32_t* uv = (int32_t*)malloc(sizeof(int32_t) * 2 * (n ? n : 1));
  float* z = (float*)malloc(sizeof(float) * (n ? n : 1));
  int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
  unsigned long long* owner = (unsigned long long*)calloc(WH, sizeof(unsigned long long));
  if (!uv || !z || !idx || !owner) { free(uv); free(z); free(idx); free(owner); return SMVS_ENOMEM; }
  size_t m = 0;
  orc_delaunay_points(v, xyz, n, uv, z, idx, &m);
  /* The depth range covers every projected point (:1251-1254). */
  float lo = FLT_MAX, hi = FLT_EPSILON;
  for (size_t k = 0; k < m; ++k) { lo = fminf(lo, z[k]); hi = fmaxf(hi, z[k]); }
  memset(depth, 0, sizeof(float) * WH);
  memset(normal, 0, sizeof(float) * 3 * WH);
  double Kd[9], Kid[9];
  for (int k = 0; k < 9; ++k) Kd[k] = v->K[k];
  inverse3d(Kd, Kid);
  float kinv[9];
  for (int k = 0; k < 9; ++k) kinv[k] = (float)Kid[k];
  for (int pass = 0; pass < 2; ++pass)
    for (size_t t = 0; t < ntri; ++t) {
      double x[3], y[3];
      float c[3][3];
      int id[3];
      for (int k = 0; k < 3; ++k) {
        id[k] = tris[3 * t + k];
        if (id[k] < 0 || (size_t)id[k] >= m) { free(uv); free(z); free(idx); free(owner); return SMVS_EINVAL; }
        x[k] = (double)uv[2 * id[k]];
        y[k] = (double)uv[2 * id[k] + 1];
        const double zz = (double)z[id[k]];
        const float q[3] = {(float)(x[k] * zz), (float)(y[k] * zz), (float)zz};
        for (int r = 0; r < 3; ++r) c[k][r] = dot3f(kinv + 3 * r, q);
      }
      const float e1[3] = {c[1][0] - c[0][0], c[1][1] - c[0][1], c[1][2] - c[0][2]};
      const float e2[3] = {c[2][0] - c[0][0], c[2][1] - c[0][1], c[2][2] - c[0][2]};
      float nn[3] = {e2[1] * e1[2] - e2[2] * e1[1], e2[2] * e1[0] - e2[0] * e1[2], e2[0] * e1[1] - e2[1] * e1[0]};
      const float sq = dot3f(nn, nn);
      if (sq > 0.0f) {
        const float nrm = sqrtf(sq);
        nn[0] = nn[0] / nrm; nn[1] = nn[1] / nrm; nn[2] = nn[2] / nrm;
      }
      const float inv = 1.0f / dot3f(nn, c[0]);
      const float np[3] = {nn[0] * inv, nn[1] * inv, nn[2] * inv};
      int a = id[0], b = id[1], e = id[2], s;
      if (a < b) { s = a; a = b; b = s; }
      if (b < e) { s = b; b = e; e = s; }
      if (a < b) { s = a; a = b; b = s; }
      const unsigned long long key =
          (((unsigned long long)a << 42) | ((unsigned long long)b << 21) | (unsigned long long)e) + 1ull;
      double umin = x[0], umax = x[0], vmin = y[0], vmax = y[0];
      for (int k = 1; k < 3; ++k) {
        umin = fmin(umin, x[k]); umax = fmax(umax, x[k]);
        vmin = fmin(vmin, y[k]); vmax = fmax(vmax, y[k]);
      }
      const int u0 = (int)umin > 0 ? (int)umin : 0, u1 = (int)umax < W - 1 ? (int)umax : W - 1;
      const int v0 = (int)vmin > 0 ? (int)vmin : 0, v1 = (int)vmax < H - 1 ? (int)vmax : H - 1;
      for (int vv = v0; vv <= v1; ++vv)
        for (int uu = u0; uu <= u1; ++uu) {
          const double m1 = (x[1] - x[0]) * ((double)vv - y[0]) - ((double)uu - x[0]) * (y[1] - y[0]);
          const double m2 = (x[2] - x[1]) * ((double)vv - y[1]) - ((double)uu - x[1]) * (y[2] - y[1]);
          const double m3 = (x[0] - x[2]) * ((double)vv - y[2]) - ((double)uu - x[2]) * (y[0] - y[2]);
          if (!(m1 >= 0 && m2 >= 0 && m3 >= 0)) continue;
          const size_t p = (size_t)vv * W + uu;
          if (pass == 0) {
            if (key > owner[p]) owner[p] = key;
            continue;
          }
          if (owner[p] != key) continue;
          const float q[3] = {(float)uu, (float)vv, 1.0f};
          float xc[3];
          for (int r = 0; r < 3; ++r) xc[r] = dot3f(kinv + 3 * r, q);
          depth[p] = 1.0f / dot3f(np, xc);
          normal[p] = nn[0];
          normal[WH + p] = nn[1];
          normal[2 * WH + p] = nn[2];
        }
    }
  finish_range(lo, hi, range);
  free(uv); free(z); free(idx); free(owner);
  return SMVS_OK;
}
