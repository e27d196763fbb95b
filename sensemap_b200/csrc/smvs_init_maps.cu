// smvs_init_maps.cu — initial depth/normal maps from the sparse or prior model.
//
// Replaces the host loops PatchMatchController runs before a PatchMatch pass
// (src/controllers/patch_match_controller.cc): InitDepthMap (:1205-1307) with
// InitDepthMapFromSparsePoint (:483-518), Model2Depth (:520-642) and Ply2Depth
// (:643-750). Each is a scatter with a depth test: candidates (a point's 7x7
// window, a triangle's covered pixels, an oriented point's odd-pixel window)
// write a pixel when the map is empty there or their depth is below the stored
// float. The reference applies the candidates one after another; here every
// candidate is a GPU thread's work and the sequential result is rebuilt from
// order-independent atomics:
//   - the stored depth is the minimum float over the pixel's candidates;
//   - the winning candidate (whose normal is stored) is the first candidate
//     with that float, unless a later one with the same float has a double
//     depth below it (the reference compares the double with the stored
//     float): then the last such one;
//   - the largest depth written anywhere (the depth range's upper end) is the
//     first candidate's depth at each pixel, since later writes only lower it.
// The float path (sparse points) writes no normals and keeps the minimum.
// Compiled without FMA contraction (double and float): the arithmetic is the
// CPU oracle's, term for term.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include <vector>

#include <cuda_runtime.h>

#include "../../include/smvs.h"

extern "C" void smvs_internal_set_error(const char* msg);
cudaMemPool_t smvs_internal_device_pool(int device);

namespace smvs {
// smvs_delaunay.cpp
int DelaunayTriangulate(const int32_t* xy, int n, std::vector<int32_t>& tris);
}

namespace {

int Fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  smvs_internal_set_error(buf);
  return code;
}

#define IM_CUDA(call)                                                                                      \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return Fail(SMVS_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// Order-preserving map float -> uint32 (for atomicMin/Max over signed floats).
__host__ __device__ __forceinline__ uint32_t FKey(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ __forceinline__ float FromKey(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

struct Cam {
  float Kf[9], Rf[9], Tf[3];     // float pose (sparse path)
  double K[9], R[9], T[3], Kinv[9], C[3], ray[3];
  int W, H;
};

// 3x3 inverse by the adjugate (oracle: inverse3d).
void Inverse3(const double* m, double* inv) {
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

Cam MakeCam(const smvs_view& v) {
  Cam c;
  memcpy(c.Kf, v.K, sizeof(c.Kf));
  memcpy(c.Rf, v.R, sizeof(c.Rf));
  memcpy(c.Tf, v.T, sizeof(c.Tf));
  for (int k = 0; k < 9; ++k) { c.K[k] = v.K[k]; c.R[k] = v.R[k]; }
  for (int k = 0; k < 3; ++k) c.T[k] = v.T[k];
  Inverse3(c.K, c.Kinv);
  for (int r = 0; r < 3; ++r) c.C[r] = -(c.R[r] * c.T[0] + c.R[3 + r] * c.T[1] + c.R[6 + r] * c.T[2]);
  for (int k = 0; k < 3; ++k) c.ray[k] = c.R[6 + k];
  c.W = v.width;
  c.H = v.height;
  return c;
}

template <typename T>
__device__ __forceinline__ void Apply3(const T* M, const T* y, const T* t, T* x) {
  for (int r = 0; r < 3; ++r) {
    const T s = M[3 * r] * y[0] + M[3 * r + 1] * y[1] + M[3 * r + 2] * y[2];
    x[r] = t ? s + t[r] : s;
  }
}
__device__ __forceinline__ double Dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// double -> int truncation for pixel bounds; values beyond +-2^30 (where the
// reference's conversion is undefined) are clamped, NaN gives -2^30.
__device__ __forceinline__ int ToInt(double x) {
  if (x != x) return -1073741824;
  return (int)fmin(fmax(x, -1073741824.0), 1073741824.0);
}

// ---------------------------------------------------------------------------
// Sparse points: InitDepthMap projection + InitDepthMapFromSparsePoint splat.
// ---------------------------------------------------------------------------
__global__ void SparseSplatKernel(Cam c, const float* __restrict__ xyz, size_t n, uint32_t* __restrict__ key,
                                  uint32_t* __restrict__ range) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float X[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    float Y[3], Xc[3];
    Apply3(c.Rf, X, c.Tf, Y);
    Apply3(c.Kf, Y, (const float*)nullptr, Xc);
    if (!(Xc[2] > 0)) continue;
    const float qu = Xc[0] / Xc[2], qv = Xc[1] / Xc[2];
    // (int) truncates toward zero; out-of-range values are rejected first.
    if (!(qu > -1.0f && qu < (float)c.W && qv > -1.0f && qv < (float)c.H)) continue;
    const int fu = (int)qu, fv = (int)qv;
    const float z = Xc[2];
    atomicMin(range, FKey(z));
    atomicMax(range + 1, FKey(z));
    const uint32_t kz = FKey(z);
    const int u0 = max(fu - 3, 0), u1 = min(fu + 3, c.W - 1), v0 = max(fv - 3, 0), v1 = min(fv + 3, c.H - 1);
    for (int y = v0; y <= v1; ++y)
      for (int x = u0; x <= u1; ++x) atomicMin(key + (size_t)y * c.W + x, kz);
  }
}

__global__ void SparseResolveKernel(const uint32_t* __restrict__ key, size_t wh, float* __restrict__ depth,
                                    float* __restrict__ normal) {
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < wh; p += (size_t)gridDim.x * blockDim.x) {
    const uint32_t k = key[p];
    depth[p] = k == 0xffffffffu ? 0.0f : FromKey(k);
    normal[p] = 0.0f;
    normal[wh + p] = 0.0f;
    normal[2 * wh + p] = 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Depth-tested scatter shared by the mesh and dense-point paths.
// ---------------------------------------------------------------------------
struct PixelState {
  uint32_t* key;     // min FKey((float)z)
  int* first;        // first candidate covering the pixel
  int* first_eq;     // first candidate whose float equals the minimum
  int* last_up;      // last candidate with that float and a double depth below it
  int* bad;          // set when a resolve pass meets an index out of range
};

// Pass 1 / pass 2 of one candidate (index `cand`, pixel p, double depth z).
__device__ __forceinline__ void Visit(const PixelState& s, int pass, int cand, size_t p, double z) {
  if (z != z) return;  // a NaN depth is never written (see the oracle)
  const float zf = (float)z;
  const uint32_t kz = FKey(zf);
  if (pass == 0) {
    atomicMin(s.key + p, kz);
    atomicMin(s.first + p, cand);
  } else if (kz == s.key[p]) {
    atomicMin(s.first_eq + p, cand);
    if (z < (double)zf) atomicMax(s.last_up + p, cand);
  }
}

// The candidate whose normal the sequential depth test leaves at pixel p:
// the first one with the minimum float, or a later one with that float whose
// double depth is below it (the last such). -1 when the state is inconsistent.
__device__ __forceinline__ int Winner(const PixelState& s, size_t p, size_t n) {
  const int w = max(s.first_eq[p], s.last_up[p]);
  if (w < 0 || (size_t)w >= n || s.first[p] < 0 || (size_t)s.first[p] >= n) {
    atomicExch(s.bad, 1);
    return -1;
  }
  return w;
}

// One triangle after Model2Depth's culling and projection (:548-591).
struct FaceRec {
  double uv[3][2];
  double np[3];   // normal / (normal . Xc0)
  double nn[3];   // camera-frame unit normal
  int u0, u1, v0, v1;  // pixel box; u0 > u1 marks a culled face
};

__global__ void FacePrepKernel(Cam c, const double* __restrict__ vert, size_t nvert, const int32_t* __restrict__ faces,
                               size_t nface, const double* __restrict__ fnorm, double thresh_fov,
                               FaceRec* __restrict__ out, int* __restrict__ bad_index) {
  for (size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x; f < nface; f += (size_t)gridDim.x * blockDim.x) {
    FaceRec r;
    r.u0 = 1;
    r.u1 = 0;
    const int32_t a = faces[3 * f], b = faces[3 * f + 1], cc = faces[3 * f + 2];
    if (a < 0 || b < 0 || cc < 0 || (size_t)a >= nvert || (size_t)b >= nvert || (size_t)cc >= nvert) {
      atomicMin(bad_index, (int)min(f, (size_t)INT_MAX));
      out[f] = r;
      continue;
    }
    const double* p[3] = {vert + 3 * (size_t)a, vert + 3 * (size_t)b, vert + 3 * (size_t)cc};
    double cen[3], d[3];
    for (int k = 0; k < 3; ++k) cen[k] = (p[0][k] + p[1][k] + p[2][k]) / 3;
    for (int k = 0; k < 3; ++k) d[k] = cen[k] - c.C[k];
    if (Dot3(d, fnorm + 3 * f) > 0) { out[f] = r; continue; }  // back face (:557-559)
    const double len = sqrt(Dot3(d, d));
    if (len > 0) for (int k = 0; k < 3; ++k) d[k] = d[k] / len;
    if (Dot3(c.ray, d) < thresh_fov) { out[f] = r; continue; }
    double Xc[3][3];
    for (int k = 0; k < 3; ++k) {
      double uvw[3];
      Apply3(c.R, p[k], c.T, Xc[k]);
      Apply3(c.K, Xc[k], (const double*)nullptr, uvw);
      const double w = uvw[2];
      r.uv[k][0] = uvw[0] / w;
      r.uv[k][1] = uvw[1] / w;
    }
    int u_min = ToInt(fmin(r.uv[0][0], fmin(r.uv[1][0], r.uv[2][0])));
    int u_max = ToInt(fmax(r.uv[0][0], fmax(r.uv[1][0], r.uv[2][0])));
    int v_min = ToInt(fmin(r.uv[0][1], fmin(r.uv[1][1], r.uv[2][1])));
    int v_max = ToInt(fmax(r.uv[0][1], fmax(r.uv[1][1], r.uv[2][1])));
    u_min = max(0, u_min);
    v_min = max(0, v_min);
    u_max = min(c.W - 1, u_max);
    v_max = min(c.H - 1, v_max);
    if (Xc[0][2] <= 0 || Xc[1][2] <= 0 || Xc[2][2] <= 0 || u_min > u_max || v_min > v_max) { out[f] = r; continue; }
    double e1[3], e2[3];
    for (int k = 0; k < 3; ++k) { e1[k] = Xc[1][k] - Xc[0][k]; e2[k] = Xc[2][k] - Xc[0][k]; }
    r.nn[0] = e1[1] * e2[2] - e1[2] * e2[1];
    r.nn[1] = e1[2] * e2[0] - e1[0] * e2[2];
    r.nn[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double nl = sqrt(Dot3(r.nn, r.nn));
    if (nl > 0) for (int k = 0; k < 3; ++k) r.nn[k] = r.nn[k] / nl;
    const double ip = 1.0 / Dot3(r.nn, Xc[0]);
    for (int k = 0; k < 3; ++k) r.np[k] = r.nn[k] * ip;
    r.u0 = u_min; r.u1 = u_max; r.v0 = v_min; r.v1 = v_max;
    out[f] = r;
  }
}

// Inside test and plane depth of one pixel (:593-608).
__device__ __forceinline__ bool FaceDepth(const FaceRec& r, const double* Kinv, int x, int y, double* z) {
  const double a1x = r.uv[1][0] - r.uv[0][0], a1y = r.uv[1][1] - r.uv[0][1];
  const double a2x = r.uv[2][0] - r.uv[1][0], a2y = r.uv[2][1] - r.uv[1][1];
  const double a3x = r.uv[0][0] - r.uv[2][0], a3y = r.uv[0][1] - r.uv[2][1];
  const double m1 = a1x * (y - r.uv[0][1]) - (x - r.uv[0][0]) * a1y;
  const double m2 = a2x * (y - r.uv[1][1]) - (x - r.uv[1][0]) * a2y;
  const double m3 = a3x * (y - r.uv[2][1]) - (x - r.uv[2][0]) * a3y;
  if (!(m1 < 0 && m2 < 0 && m3 < 0)) return false;
  const double pix[3] = {(double)x, (double)y, 1.0};
  double xc[3];
  Apply3(Kinv, pix, (const double*)nullptr, xc);
  *z = 1.0 / Dot3(r.np, xc);
  return true;
}

__global__ void FaceScatterKernel(Cam c, const FaceRec* __restrict__ recs, size_t nface, PixelState s, int pass) {
  for (size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x; f < nface; f += (size_t)gridDim.x * blockDim.x) {
    const FaceRec r = recs[f];
    if (r.u0 > r.u1) continue;
    for (int y = r.v0; y <= r.v1; ++y)
      for (int x = r.u0; x <= r.u1; ++x) {
        double z;
        if (FaceDepth(r, c.Kinv, x, y, &z)) Visit(s, pass, (int)f, (size_t)y * c.W + x, z);
      }
  }
}

__global__ void FaceResolveKernel(Cam c, const FaceRec* __restrict__ recs, size_t nface, PixelState s,
                                  float* __restrict__ depth, float* __restrict__ normal, uint32_t* __restrict__ range) {
  const size_t wh = (size_t)c.W * c.H;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < wh; p += (size_t)gridDim.x * blockDim.x) {
    const int first = s.first[p];
    const int win = first == INT_MAX ? -1 : Winner(s, p, nface);
    if (win < 0) {
      depth[p] = 0.0f;
      normal[p] = normal[wh + p] = normal[2 * wh + p] = 0.0f;
      continue;
    }
    const float d = FromKey(s.key[p]);
    depth[p] = d;
    normal[p] = (float)recs[win].nn[0];
    normal[wh + p] = (float)recs[win].nn[1];
    normal[2 * wh + p] = (float)recs[win].nn[2];
    double z0 = 0.0;
    FaceDepth(recs[first], c.Kinv, (int)(p % c.W), (int)(p / c.W), &z0);
    atomicMin(range, FKey(d));
    atomicMax(range + 1, FKey((float)z0));
  }
}

// Ply2Depth candidates of one oriented point (:660-725).
struct PointRec {
  double z;            // Xc[2]
  float n[3];          // R * normal, as stored
  int i0, i1, j0, j1;  // window; i0 > i1 marks a culled point
};

__global__ void PointPrepKernel(Cam c, const float* __restrict__ xyz, const float* __restrict__ nrm, size_t n, int ws,
                                PointRec* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    PointRec r;
    r.i0 = 1;
    r.i1 = 0;
    const double cen[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    const double nw[3] = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
    double inrm[3], d[3], Xc[3], uv[3];
    Apply3(c.R, nw, (const double*)nullptr, inrm);
    for (int k = 0; k < 3; ++k) d[k] = cen[k] - c.C[k];
    if (Dot3(d, nw) > 0) { out[i] = r; continue; }
    Apply3(c.R, cen, c.T, Xc);
    Apply3(c.K, Xc, (const double*)nullptr, uv);
    uv[0] = uv[0] / uv[2];
    uv[1] = uv[1] / uv[2];
    if (Xc[2] <= 0 || !(uv[0] >= 0 && uv[1] >= 0 && uv[0] <= c.W - 1 && uv[1] <= c.H - 1)) {  // NaN too
      out[i] = r;
      continue;
    }
    r.z = Xc[2];
    for (int k = 0; k < 3; ++k) r.n[k] = (float)inrm[k];
    r.i0 = (int)floor(uv[0]) - ws;
    r.i1 = (int)ceil(uv[0]) + ws;
    r.j0 = (int)floor(uv[1]) - ws;
    r.j1 = (int)ceil(uv[1]) + ws;
    out[i] = r;
  }
}

__global__ void PointScatterKernel(Cam c, const PointRec* __restrict__ recs, size_t n, PixelState s, int pass) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const PointRec r = recs[i];
    if (r.i0 > r.i1) continue;
    for (int x = max(r.i0, 0); x <= min(r.i1, c.W - 1); ++x) {
      if (x % 2 == 0) continue;  // odd columns and rows only (:707-709)
      for (int y = max(r.j0, 0); y <= min(r.j1, c.H - 1); ++y)
        if (y % 2 != 0) Visit(s, pass, (int)i, (size_t)y * c.W + x, r.z);
    }
  }
}

__global__ void PointResolveKernel(Cam c, const PointRec* __restrict__ recs, size_t npoint, PixelState s,
                                   float* __restrict__ depth, float* __restrict__ normal,
                                   uint32_t* __restrict__ range) {
  const size_t wh = (size_t)c.W * c.H;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < wh; p += (size_t)gridDim.x * blockDim.x) {
    const int first = s.first[p];
    const int win = first == INT_MAX ? -1 : Winner(s, p, npoint);
    if (win < 0) {
      depth[p] = 0.0f;
      normal[p] = normal[wh + p] = normal[2 * wh + p] = 0.0f;
      continue;
    }
    const float d = FromKey(s.key[p]);
    depth[p] = d;
    normal[p] = recs[win].n[0];
    normal[wh + p] = recs[win].n[1];
    normal[2 * wh + p] = recs[win].n[2];
    atomicMin(range, FKey(d));
    atomicMax(range + 1, FKey((float)recs[first].z));
  }
}

// ---------------------------------------------------------------------------
// Delaunay initial map: InitDepthMap's projection (:1236-1256, truncated pixel
// positions), then InitDepthMapFromDelaunay (:398-474) over the triangulation
// of those positions: each triangle's plane through its three back-projected
// points is written, depth and camera-frame normal, to the pixels inside it.
// ---------------------------------------------------------------------------
__global__ void ProjectUvdKernel(Cam c, const float* __restrict__ xyz, size_t n, int2* __restrict__ uv,
                                 float* __restrict__ z, uint32_t* __restrict__ range) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float X[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    float Y[3], Xc[3];
    Apply3(c.Rf, X, c.Tf, Y);
    Apply3(c.Kf, Y, (const float*)nullptr, Xc);
    uv[i] = make_int2(-1, -1);
    if (!(Xc[2] > 0)) continue;
    const float qu = Xc[0] / Xc[2], qv = Xc[1] / Xc[2];
    if (!(qu > -1.0f && qu < (float)c.W && qv > -1.0f && qv < (float)c.H)) continue;
    uv[i] = make_int2((int)qu, (int)qv);
    z[i] = Xc[2];
    atomicMin(range, FKey(Xc[2]));
    atomicMax(range + 1, FKey(Xc[2]));
  }
}

struct DelaunayTri {
  double x[3], y[3];  // vertex positions (pixels, as the reference's double CGAL points)
  float n[3];         // unit normal (edge2 x edge1)
  float np[3];        // normal / (normal . c0)
  int u0, u1, v0, v1; // pixel box, clipped to the image
  unsigned long long key;  // order-free owner key of shared pixels (0 = degenerate, skipped)
};

__device__ __forceinline__ float Dot3f(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

// Per triangle: the plane of RasterDepthDataPlaneData (:230-247) from the
// three points (u z, v z, z) mapped by K^-1 (float), as :435-447 composes it.
__global__ void DelaunayPrepKernel(const int2* __restrict__ uv, const float* __restrict__ z,
                                   const int32_t* __restrict__ vid, const int32_t* __restrict__ tris, int ntri,
                                   const float* __restrict__ kinv, int W, int H, DelaunayTri* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  DelaunayTri d;
  float c[3][3];
  int idx[3];
  for (int k = 0; k < 3; ++k) {
    idx[k] = tris[3 * t + k];
    const int p = vid[idx[k]];
    d.x[k] = (double)uv[p].x;
    d.y[k] = (double)uv[p].y;
    const double zz = (double)z[p];
    const float q[3] = {(float)(d.x[k] * zz), (float)(d.y[k] * zz), (float)zz};
    for (int r = 0; r < 3; ++r) c[k][r] = Dot3f(kinv + 3 * r, q);
  }
  const float e1[3] = {c[1][0] - c[0][0], c[1][1] - c[0][1], c[1][2] - c[0][2]};
  const float e2[3] = {c[2][0] - c[0][0], c[2][1] - c[0][1], c[2][2] - c[0][2]};
  float nn[3] = {e2[1] * e1[2] - e2[2] * e1[1], e2[2] * e1[0] - e2[0] * e1[2], e2[0] * e1[1] - e2[1] * e1[0]};
  const float sq = Dot3f(nn, nn);
  if (sq > 0.0f) {  // Eigen's normalized(): divide by the norm when it is not 0
    const float nrm = sqrtf(sq);
    nn[0] = nn[0] / nrm; nn[1] = nn[1] / nrm; nn[2] = nn[2] / nrm;
  }
  const float inv = 1.0f / Dot3f(nn, c[0]);
  for (int r = 0; r < 3; ++r) { d.n[r] = nn[r]; d.np[r] = nn[r] * inv; }
  const double umin = fmin(d.x[0], fmin(d.x[1], d.x[2])), umax = fmax(d.x[0], fmax(d.x[1], d.x[2]));
  const double vmin = fmin(d.y[0], fmin(d.y[1], d.y[2])), vmax = fmax(d.y[0], fmax(d.y[1], d.y[2]));
  d.u0 = max(0, (int)umin); d.u1 = min(W - 1, (int)umax);
  d.v0 = max(0, (int)vmin); d.v1 = min(H - 1, (int)vmax);
  // A pixel on an edge shared by two triangles is written by both in the
  // reference, the later face in CGAL's face order last. The triangle with the
  // largest sorted vertex triple writes it here, whatever the list order.
  int a = idx[0], b = idx[1], e = idx[2];
  if (a < b) { const int t2 = a; a = b; b = t2; }
  if (b < e) { const int t2 = b; b = e; e = t2; }
  if (a < b) { const int t2 = a; a = b; b = t2; }
  d.key = ((unsigned long long)a << 42) | ((unsigned long long)b << 21) | (unsigned long long)e;
  d.key += 1ull;
  out[t] = d;
}

__device__ __forceinline__ bool InsideTri(const DelaunayTri& d, int u, int v) {
  // :451-461 with Vector2d edges v1 = i1 - i0, v2 = i2 - i1, v3 = i0 - i2.
  const double m1 = (d.x[1] - d.x[0]) * ((double)v - d.y[0]) - ((double)u - d.x[0]) * (d.y[1] - d.y[0]);
  const double m2 = (d.x[2] - d.x[1]) * ((double)v - d.y[1]) - ((double)u - d.x[1]) * (d.y[2] - d.y[1]);
  const double m3 = (d.x[0] - d.x[2]) * ((double)v - d.y[2]) - ((double)u - d.x[2]) * (d.y[0] - d.y[2]);
  return m1 >= 0 && m2 >= 0 && m3 >= 0;
}

__global__ void DelaunayClaimKernel(const DelaunayTri* __restrict__ tri, int ntri, int W,
                                    unsigned long long* __restrict__ owner) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  const DelaunayTri d = tri[t];
  for (int v = d.v0; v <= d.v1; ++v)
    for (int u = d.u0; u <= d.u1; ++u)
      if (InsideTri(d, u, v)) atomicMax(owner + (size_t)v * W + u, d.key);
}

__global__ void DelaunayWriteKernel(const DelaunayTri* __restrict__ tri, int ntri, int W, int H,
                                    const unsigned long long* __restrict__ owner, const float* __restrict__ kinv,
                                    float* __restrict__ depth, float* __restrict__ normal) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  const DelaunayTri d = tri[t];
  const size_t wh = (size_t)W * H;
  for (int v = d.v0; v <= d.v1; ++v)
    for (int u = d.u0; u <= d.u1; ++u) {
      const size_t p = (size_t)v * W + u;
      if (owner[p] != d.key || !InsideTri(d, u, v)) continue;
      const float q[3] = {(float)u, (float)v, 1.0f};
      float xc[3];
      for (int r = 0; r < 3; ++r) xc[r] = Dot3f(kinv + 3 * r, q);
      depth[p] = 1.0f / Dot3f(d.np, xc);
      normal[p] = d.n[0];
      normal[wh + p] = d.n[1];
      normal[2 * wh + p] = d.n[2];
    }
}

__global__ void FillKernel(uint32_t* __restrict__ p, size_t n, uint32_t v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

int Grid(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

// Scratch and host/device plumbing of one call.
struct Call {
  cudaStream_t stream;
  cudaMemPool_t pool;
  int memory;
  void* blocks[16] = {};
  int nblocks = 0;
  ~Call() {
    for (int k = 0; k < nblocks; ++k) cudaFreeAsync(blocks[k], stream);
  }
  template <typename T>
  int Alloc(T** p, size_t bytes) {
    if (nblocks == (int)(sizeof(blocks) / sizeof(blocks[0]))) return Fail(SMVS_ENOMEM, "init maps: too many buffers");
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), std::max<size_t>(bytes, 16), pool, stream);
    if (e != cudaSuccess) return Fail(SMVS_ENOMEM, "init maps: device allocation of %zu bytes: %s", bytes,
                                      cudaGetErrorString(e));
    blocks[nblocks++] = *p;
    return SMVS_OK;
  }
  // A device view of caller input: the pointer itself, or a copy of host memory.
  template <typename T>
  int In(const T* src, size_t count, const T** out) {
    if (memory == SMVS_MEM_DEVICE || count == 0) { *out = src; return SMVS_OK; }
    T* d;
    int st = Alloc(&d, count * sizeof(T));
    if (st) return st;
    IM_CUDA(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, stream));
    *out = d;
    return SMVS_OK;
  }
};

int Check(const smvs_view* view, int memory, float* depth, float* normal) {
  if (!view || !depth || !normal) return Fail(SMVS_EINVAL, "init maps: null argument");
  if (memory != SMVS_MEM_HOST && memory != SMVS_MEM_DEVICE) return Fail(SMVS_EINVAL, "init maps: bad memory kind");
  if (view->width < 1 || view->height < 1 || (size_t)view->width * view->height >= ((size_t)1 << 31))
    return Fail(SMVS_EINVAL, "init maps: bad view size %dx%d", view->width, view->height);
  return SMVS_OK;
}

// After the arguments are checked: the device's pool and the caller's stream.
int Begin(int memory, void* stream, Call* call) {
  int dev = 0;
  IM_CUDA(cudaGetDevice(&dev));
  call->stream = (cudaStream_t)stream;
  call->memory = memory;
  call->pool = smvs_internal_device_pool(dev);
  if (!call->pool) return Fail(SMVS_ECUDA, "init maps: no memory pool on device %d", dev);
  return SMVS_OK;
}

// Output maps (device) and the final copy for host callers; the depth range
// (optional) is read back, which waits for the stream.
int Finish(Call* call, const smvs_view* view, float* d_depth, float* d_normal, float* depth, float* normal,
           const uint32_t* d_range, float* depth_range, bool has_range) {
  const size_t wh = (size_t)view->width * view->height;
  if (call->memory == SMVS_MEM_HOST) {
    IM_CUDA(cudaMemcpyAsync(depth, d_depth, wh * 4, cudaMemcpyDeviceToHost, call->stream));
    IM_CUDA(cudaMemcpyAsync(normal, d_normal, wh * 12, cudaMemcpyDeviceToHost, call->stream));
  }
  uint32_t r[2] = {0xffffffffu, 0};
  if (has_range && depth_range) IM_CUDA(cudaMemcpyAsync(r, d_range, 8, cudaMemcpyDeviceToHost, call->stream));
  if (call->memory == SMVS_MEM_HOST || (has_range && depth_range)) IM_CUDA(cudaStreamSynchronize(call->stream));
  if (depth_range) {
    // :1297-1304: no write keeps (FLT_MAX, FLT_EPSILON) -> (0, 100); then
    // first *= 0.9 is overwritten by 1e-6 and second *= 1.1.
    const float lo = FromKey(r[0]);
    const float hi = FromKey(r[1]);
    depth_range[0] = 0.000001f;
    depth_range[1] = (lo == FLT_MAX ? 100.0f : hi) * 1.1f;
  }
  return SMVS_OK;
}

int Outputs(Call* call, const smvs_view* view, float* depth, float* normal, float** d_depth, float** d_normal) {
  const size_t wh = (size_t)view->width * view->height;
  if (call->memory == SMVS_MEM_DEVICE) {
    *d_depth = depth;
    *d_normal = normal;
    return SMVS_OK;
  }
  int st = call->Alloc(d_depth, wh * 4);
  if (!st) st = call->Alloc(d_normal, wh * 12);
  return st;
}

int PixelScratch(Call* call, size_t wh, PixelState* s, uint32_t** range) {
  int st = call->Alloc(&s->key, wh * 4);
  if (!st) st = call->Alloc(&s->first, wh * 4);
  if (!st) st = call->Alloc(&s->first_eq, wh * 4);
  if (!st) st = call->Alloc(&s->last_up, wh * 4);
  if (!st) st = call->Alloc(&s->bad, 4);
  if (!st) st = call->Alloc(range, 8);
  if (st) return st;
  IM_CUDA(cudaMemsetAsync(s->bad, 0, 4, call->stream));
  FillKernel<<<Grid(wh), 256, 0, call->stream>>>(s->key, wh, 0xffffffffu);
  FillKernel<<<Grid(wh), 256, 0, call->stream>>>(reinterpret_cast<uint32_t*>(s->first), wh, (uint32_t)INT_MAX);
  FillKernel<<<Grid(wh), 256, 0, call->stream>>>(reinterpret_cast<uint32_t*>(s->first_eq), wh, (uint32_t)INT_MAX);
  IM_CUDA(cudaMemsetAsync(s->last_up, 0xff, wh * 4, call->stream));  // -1
  const uint32_t r0[2] = {FKey(FLT_MAX), FKey(FLT_EPSILON)};
  IM_CUDA(cudaMemcpyAsync(*range, r0, 8, cudaMemcpyHostToDevice, call->stream));
  IM_CUDA(cudaGetLastError());
  return SMVS_OK;
}

}  // namespace

extern "C" {

int smvs_init_depth_from_sparse_points(const smvs_view* view, const float* xyz, size_t num_points, int memory,
                                       float* depth, float* normal, float* depth_range, void* stream) {
  int st = Check(view, memory, depth, normal);
  if (st) return st;
  if (num_points && !xyz) return Fail(SMVS_EINVAL, "init maps: null points");
  Call call;
  if ((st = Begin(memory, stream, &call))) return st;
  const size_t wh = (size_t)view->width * view->height;
  const float* d_xyz;
  float *d_depth, *d_normal;
  uint32_t *key, *range;
  if ((st = call.In(xyz, num_points * 3, &d_xyz))) return st;
  if ((st = Outputs(&call, view, depth, normal, &d_depth, &d_normal))) return st;
  if ((st = call.Alloc(&key, wh * 4)) || (st = call.Alloc(&range, 8))) return st;
  const Cam c = MakeCam(*view);
  FillKernel<<<Grid(wh), 256, 0, call.stream>>>(key, wh, 0xffffffffu);
  const uint32_t r0[2] = {FKey(FLT_MAX), FKey(FLT_EPSILON)};
  IM_CUDA(cudaMemcpyAsync(range, r0, 8, cudaMemcpyHostToDevice, call.stream));
  if (num_points) SparseSplatKernel<<<Grid(num_points), 256, 0, call.stream>>>(c, d_xyz, num_points, key, range);
  SparseResolveKernel<<<Grid(wh), 256, 0, call.stream>>>(key, wh, d_depth, d_normal);
  IM_CUDA(cudaGetLastError());
  return Finish(&call, view, d_depth, d_normal, depth, normal, range, depth_range, true);
}

int smvs_init_depth_from_delaunay(const smvs_view* view, const float* xyz, size_t num_points, int memory,
                                  float* depth, float* normal, float* depth_range, void* stream) {
  int st = Check(view, memory, depth, normal);
  if (st) return st;
  if (num_points && !xyz) return Fail(SMVS_EINVAL, "init maps: null points");
  if (num_points >= ((size_t)1 << 21)) return Fail(SMVS_EINVAL, "init maps: at most 2^21 - 1 points per view");
  Call call;
  if ((st = Begin(memory, stream, &call))) return st;
  const size_t wh = (size_t)view->width * view->height;
  const float* d_xyz;
  float *d_depth, *d_normal, *d_z;
  int2* d_uv;
  uint32_t* range;
  if ((st = call.In(xyz, num_points * 3, &d_xyz))) return st;
  if ((st = Outputs(&call, view, depth, normal, &d_depth, &d_normal))) return st;
  if ((st = call.Alloc(&d_uv, std::max<size_t>(num_points, 1) * sizeof(int2))) ||
      (st = call.Alloc(&d_z, std::max<size_t>(num_points, 1) * sizeof(float))) || (st = call.Alloc(&range, 8)))
    return st;
  const Cam c = MakeCam(*view);
  const uint32_t r0[2] = {FKey(FLT_MAX), FKey(FLT_EPSILON)};
  IM_CUDA(cudaMemcpyAsync(range, r0, 8, cudaMemcpyHostToDevice, call.stream));
  IM_CUDA(cudaMemsetAsync(d_depth, 0, wh * 4, call.stream));
  IM_CUDA(cudaMemsetAsync(d_normal, 0, wh * 12, call.stream));
  std::vector<int2> uv(num_points);
  if (num_points) {
    ProjectUvdKernel<<<Grid(num_points), 256, 0, call.stream>>>(c, d_xyz, num_points, d_uv, d_z, range);
    IM_CUDA(cudaGetLastError());
    IM_CUDA(cudaMemcpyAsync(uv.data(), d_uv, num_points * sizeof(int2), cudaMemcpyDeviceToHost, call.stream));
    IM_CUDA(cudaStreamSynchronize(call.stream));
  }
  // The points that landed in the image, in input order, and the Delaunay
  // triangulation of their pixel positions (host).
  std::vector<int32_t> vid, xy, tris;
  for (size_t i = 0; i < num_points; ++i)
    if (uv[i].x >= 0) {
      vid.push_back((int32_t)i);
      xy.push_back(uv[i].x);
      xy.push_back(uv[i].y);
    }
  if ((st = smvs::DelaunayTriangulate(xy.data(), (int)vid.size(), tris))) return st;
  const int ntri = (int)(tris.size() / 3);
  if (ntri > 0) {
    float kinv[9];
    for (int k = 0; k < 9; ++k) kinv[k] = (float)c.Kinv[k];
    int32_t *d_vid, *d_tris;
    float* d_kinv;
    DelaunayTri* d_tri;
    unsigned long long* owner;
    if ((st = call.Alloc(&d_vid, vid.size() * 4)) || (st = call.Alloc(&d_tris, tris.size() * 4)) ||
        (st = call.Alloc(&d_kinv, sizeof(kinv))) || (st = call.Alloc(&d_tri, (size_t)ntri * sizeof(DelaunayTri))) ||
        (st = call.Alloc(&owner, wh * sizeof(unsigned long long))))
      return st;
    IM_CUDA(cudaMemcpyAsync(d_vid, vid.data(), vid.size() * 4, cudaMemcpyHostToDevice, call.stream));
    IM_CUDA(cudaMemcpyAsync(d_tris, tris.data(), tris.size() * 4, cudaMemcpyHostToDevice, call.stream));
    IM_CUDA(cudaMemcpyAsync(d_kinv, kinv, sizeof(kinv), cudaMemcpyHostToDevice, call.stream));
    IM_CUDA(cudaMemsetAsync(owner, 0, wh * sizeof(unsigned long long), call.stream));
    const int blocks = (ntri + 127) / 128;
    DelaunayPrepKernel<<<blocks, 128, 0, call.stream>>>(d_uv, d_z, d_vid, d_tris, ntri, d_kinv, view->width,
                                                         view->height, d_tri);
    DelaunayClaimKernel<<<blocks, 128, 0, call.stream>>>(d_tri, ntri, view->width, owner);
    DelaunayWriteKernel<<<blocks, 128, 0, call.stream>>>(d_tri, ntri, view->width, view->height, owner, d_kinv,
                                                          d_depth, d_normal);
    IM_CUDA(cudaGetLastError());
    // The host vectors die at return: the uploads must be done first.
    IM_CUDA(cudaStreamSynchronize(call.stream));
  }
  return Finish(&call, view, d_depth, d_normal, depth, normal, range, depth_range, true);
}

int smvs_init_depth_from_mesh(const smvs_view* view, const double* vertices, size_t num_vertices,
                              const int32_t* faces, size_t num_faces, const double* face_normals, int memory,
                              float* depth, float* normal, float* depth_range, void* stream) {
  int st = Check(view, memory, depth, normal);
  if (st) return st;
  if (num_faces && (!vertices || !faces || !face_normals)) return Fail(SMVS_EINVAL, "init maps: null mesh arrays");
  if (num_faces > (size_t)INT_MAX - 1) return Fail(SMVS_EINVAL, "init maps: too many faces");
  Call call;
  if ((st = Begin(memory, stream, &call))) return st;
  const size_t wh = (size_t)view->width * view->height;
  const double *d_vert, *d_fn;
  const int32_t* d_faces;
  float *d_depth, *d_normal;
  FaceRec* recs;
  int* bad;
  PixelState s;
  uint32_t* range;
  if ((st = call.In(vertices, num_vertices * 3, &d_vert)) || (st = call.In(faces, num_faces * 3, &d_faces)) ||
      (st = call.In(face_normals, num_faces * 3, &d_fn)))
    return st;
  if ((st = Outputs(&call, view, depth, normal, &d_depth, &d_normal))) return st;
  if ((st = call.Alloc(&recs, num_faces * sizeof(FaceRec))) || (st = call.Alloc(&bad, 4))) return st;
  if ((st = PixelScratch(&call, wh, &s, &range))) return st;
  const int no_bad = INT_MAX;
  IM_CUDA(cudaMemcpyAsync(bad, &no_bad, 4, cudaMemcpyHostToDevice, call.stream));
  const Cam c = MakeCam(*view);
  if (num_faces) {
    FacePrepKernel<<<Grid(num_faces), 256, 0, call.stream>>>(c, d_vert, num_vertices, d_faces, num_faces, d_fn,
                                                             cos(90.0) /* [quirk] :536, radians */, recs, bad);
    FaceScatterKernel<<<Grid(num_faces), 256, 0, call.stream>>>(c, recs, num_faces, s, 0);
    FaceScatterKernel<<<Grid(num_faces), 256, 0, call.stream>>>(c, recs, num_faces, s, 1);
  }
  FaceResolveKernel<<<Grid(wh), 256, 0, call.stream>>>(c, recs, num_faces, s, d_depth, d_normal, range);
  IM_CUDA(cudaGetLastError());
  int bad_h = INT_MAX, state_h = 0;
  IM_CUDA(cudaMemcpyAsync(&bad_h, bad, 4, cudaMemcpyDeviceToHost, call.stream));
  IM_CUDA(cudaMemcpyAsync(&state_h, s.bad, 4, cudaMemcpyDeviceToHost, call.stream));
  st = Finish(&call, view, d_depth, d_normal, depth, normal, range, depth_range, true);
  if (st) return st;
  IM_CUDA(cudaStreamSynchronize(call.stream));
  if (bad_h != INT_MAX) return Fail(SMVS_EINVAL, "init maps: face %d indexes a missing vertex", bad_h);
  if (state_h) return Fail(SMVS_ECUDA, "init maps: inconsistent depth-test state");
  return SMVS_OK;
}

int smvs_init_depth_from_dense_points(const smvs_view* view, const float* xyz, const float* normals,
                                      size_t num_points, int level, int memory, float* depth, float* normal,
                                      float* depth_range, void* stream) {
  int st = Check(view, memory, depth, normal);
  if (st) return st;
  if (num_points && (!xyz || !normals)) return Fail(SMVS_EINVAL, "init maps: null points");
  if (level < 0 || level > 8) return Fail(SMVS_EINVAL, "init maps: level must be 0..8");
  if (num_points > (size_t)INT_MAX - 1) return Fail(SMVS_EINVAL, "init maps: too many points");
  Call call;
  if ((st = Begin(memory, stream, &call))) return st;
  const size_t wh = (size_t)view->width * view->height;
  const float *d_xyz, *d_n;
  float *d_depth, *d_normal;
  PointRec* recs;
  PixelState s;
  uint32_t* range;
  if ((st = call.In(xyz, num_points * 3, &d_xyz)) || (st = call.In(normals, num_points * 3, &d_n))) return st;
  if ((st = Outputs(&call, view, depth, normal, &d_depth, &d_normal))) return st;
  if ((st = call.Alloc(&recs, num_points * sizeof(PointRec)))) return st;
  if ((st = PixelScratch(&call, wh, &s, &range))) return st;
  const Cam c = MakeCam(*view);
  if (num_points) {
    PointPrepKernel<<<Grid(num_points), 256, 0, call.stream>>>(c, d_xyz, d_n, num_points, 1 << level, recs);
    PointScatterKernel<<<Grid(num_points), 256, 0, call.stream>>>(c, recs, num_points, s, 0);
    PointScatterKernel<<<Grid(num_points), 256, 0, call.stream>>>(c, recs, num_points, s, 1);
  }
  PointResolveKernel<<<Grid(wh), 256, 0, call.stream>>>(c, recs, num_points, s, d_depth, d_normal, range);
  IM_CUDA(cudaGetLastError());
  int state_h = 0;
  IM_CUDA(cudaMemcpyAsync(&state_h, s.bad, 4, cudaMemcpyDeviceToHost, call.stream));
  st = Finish(&call, view, d_depth, d_normal, depth, normal, range, depth_range, true);
  if (st) return st;
  IM_CUDA(cudaStreamSynchronize(call.stream));
  if (state_h) return Fail(SMVS_ECUDA, "init maps: inconsistent depth-test state");
  return SMVS_OK;
}

}  // extern "C"
