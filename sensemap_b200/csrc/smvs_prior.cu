// smvs_prior.cu — initial maps of the propagate-depth mode: the source views'
// depth maps projected into the reference view, their per-pixel median as the
// initial depth and prior depth, and normals fitted to the result
// (PatchMatchACMMCuda::InitWorkspace, patch_match_cuda.cu:603-659).
//
// Compiled with IEEE single precision (no FMA contraction, correctly rounded
// division and square root) so that the CPU oracle performs exactly the same
// operations; the reference is built with --use_fast_math, so its reciprocals
// and rsqrtf differ from these by a few units in the last place.
#include <cfloat>
#include <cstdint>
#include <cstring>

#include "smvs_kernels.h"

namespace smvs {

namespace {

// GenerateProjectDepthMaps, kernel_functions.cu:778-826: every pixel of the
// sources' common grid (the largest source width and height) lifts source v's
// depth to a world point and projects it into the reference view; the nearest
// camera depth per reference pixel wins (atomicMin on the float's bits, which
// orders positive floats). The reference reads the depth through a linear
// texture (border 0) at the integer coordinate itself, i.e. the mean of the
// four texels around the pixel corner with weights of exactly 1/4; here that
// mean is formed from the texels in double and rounded once (the hardware
// filter rounds its sum differently in the last place of some pixels).
__device__ __forceinline__ float TexelOrZero(const float* __restrict__ d, size_t pitch, int w, int h, int x, int y) {
  return (x >= 0 && x < w && y >= 0 && y < h) ? *((const float*)((const char*)d + pitch * y) + x) : 0.0f;
}

__global__ void ProjectDepthKernel(const float* __restrict__ sdepth, size_t spitch, int sw, int sh,
                                   const float* __restrict__ pose, int grid_w, int grid_h, int W, int H, float k0,
                                   float k1, float k2, float k3, unsigned int* __restrict__ composite) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= grid_w || row >= grid_h) return;
  const double sum = (double)TexelOrZero(sdepth, spitch, sw, sh, col - 1, row - 1) +
                     (double)TexelOrZero(sdepth, spitch, sw, sh, col, row - 1) +
                     (double)TexelOrZero(sdepth, spitch, sw, sh, col - 1, row) +
                     (double)TexelOrZero(sdepth, spitch, sw, sh, col, row);
  const float depth = (float)(sum * 0.25);
  if (depth < 1e-6f) return;
  const float* iP = pose + 31;  // P^-1, 3x4 row-major
  // [quirk] kernel_functions.cu:803-804 stores the products back into the int
  // pixel indices (col *= depth), truncating them toward zero.
  const float c = (float)(int)((float)col * depth), r = (float)(int)((float)row * depth);
  const float bx = iP[0] * c + iP[1] * r + iP[2] * depth + iP[3];
  const float by = iP[4] * c + iP[5] * r + iP[6] * depth + iP[7];
  const float bz = iP[8] * c + iP[9] * r + iP[10] * depth + iP[11];
  const float ibz = 1.0f / bz;
  const float bcol = ibz * k0 * bx + k1;
  const float brow = ibz * k2 * by + k3;
  // A NaN coordinate is skipped (the reference converts it to an index).
  if (!(bcol >= 0.0f && bcol < (float)W && brow >= 0.0f && brow < (float)H)) return;
  const size_t q = (size_t)(int)brow * W + (size_t)(int)bcol;
  atomicMin(composite + q, __float_as_uint(bz));
}

// CompositeInitDepthMap, kernel_functions.cu:827-862: a pixel without a
// depth (<= 0) takes the median of its projected depths when there are more
// than two, and that median becomes its prior depth when more than two
// projections lie within 1 % of it; with one or two projections it takes the
// first, or the smaller of the first two (in source order).
__global__ void CompositeDepthKernel(const float* __restrict__ composite, int N, int W, int H,
                                     float* __restrict__ depth, float* __restrict__ prior) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= W || row >= H) return;
  const size_t WH = (size_t)W * H, pix = (size_t)row * W + col;
  if (depth[pix] > 0) return;
  float d[SMVS_MAX_SRC];
  int n = 0;
  for (int i = 0; i < N; ++i) {
    const float v = composite[(size_t)i * WH + pix];
    if (v > 0 && v < FLT_MAX) d[n++] = v;
  }
  if (n > 2) {
    for (int i = 0; i < n - 1; ++i)  // BubbleSort, utils.h
      for (int j = 0; j < n - 1 - i; ++j)
        if (d[j] > d[j + 1]) { const float t = d[j]; d[j] = d[j + 1]; d[j + 1] = t; }
    const float m = d[n / 2];
    depth[pix] = m;
    int consistent = 0;
    for (int i = 0; i < n; ++i) consistent += ((double)(fabsf(d[i] - m) / m) <= 0.01) ? 1 : 0;
    if (consistent > 2) prior[pix] = m;
  } else if (n > 0) {
    depth[pix] = (n > 1) ? fminf(d[0], d[1]) : d[0];
  }
}

// EstimatePatchNormal, kernel_functions.cu:864-909: the normal of the plane
// through the four 4-neighbours of (row, col), if each is within 2 % of the
// centre's depth.
__device__ bool PatchNormal(const float* __restrict__ depth, int W, int H, int row, int col, const float iK[4],
                            float n[3]) {
  if (col >= W - 1 || row >= H - 1 || col <= 0 || row <= 0) return false;
  const float d = depth[(size_t)row * W + col];
  if (d <= 0) return false;
  const int nr[4] = {row - 1, row, row + 1, row};
  const int nc[4] = {col, col + 1, col, col - 1};
  float p[4][3];
  for (int k = 0; k < 4; ++k) {
    const float nd = depth[(size_t)nr[k] * W + nc[k]];
    if ((double)(fabsf(nd - d) / d) > 0.02) return false;
    // ComputePointAtDepth, kernel_functions.cu:308-315.
    p[k][0] = nd * (iK[0] * (float)nc[k] + iK[1]);
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
  return true;
}

// CompositeInitNormalMap, kernel_functions.cu:911-966: the component-wise
// median of the patch normals at the pixel and its four diagonal neighbours,
// re-normalised; pixels without any keep their normal.
__global__ void CompositeNormalKernel(const float* __restrict__ depth, int W, int H, float i0, float i1, float i2,
                                      float i3, float* __restrict__ normal) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= W || row >= H) return;
  const float iK[4] = {i0, i1, i2, i3};
  const int dr[5] = {0, -1, -1, 1, 1}, dc[5] = {0, -1, 1, 1, -1};
  float c[3][5];
  int n = 0;
  for (int k = 0; k < 5; ++k) {
    float e[3];
    if (PatchNormal(depth, W, H, row + dr[k], col + dc[k], iK, e)) {
      c[0][n] = e[0]; c[1][n] = e[1]; c[2][n] = e[2];
      n++;
    }
  }
  if (n == 0) return;
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < n - 1; ++i)
      for (int j = 0; j < n - 1 - i; ++j)
        if (c[a][j] > c[a][j + 1]) { const float t = c[a][j]; c[a][j] = c[a][j + 1]; c[a][j + 1] = t; }
  const int m = n >> 1;
  float v[3] = {c[0][m], c[1][m], c[2][m]};
  const float inv = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const size_t WH = (size_t)W * H, pix = (size_t)row * W + col;
  normal[pix] = v[0] * inv;
  normal[WH + pix] = v[1] * inv;
  normal[2 * WH + pix] = v[2] * inv;
}

__global__ void FillU32Kernel(unsigned int* __restrict__ out, size_t n, unsigned int value) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = value;
}

}  // namespace

cudaError_t LaunchPropagateInit(const JobParams& p, const int* src_w, const int* src_h, const float* const* src_depth,
                                const size_t* src_pitch, float* composite, float* prior, cudaStream_t stream) {
  const size_t WH = (size_t)p.W * p.H;
  int gw = 0, gh = 0;  // the sources' common grid (patch_match_cuda.cu:606-620)
  for (int i = 0; i < p.N; ++i) {
    gw = src_w[i] > gw ? src_w[i] : gw;
    gh = src_h[i] > gh ? src_h[i] : gh;
  }
  unsigned int flt_max_bits;
  const float fm = FLT_MAX;
  memcpy(&flt_max_bits, &fm, sizeof(fm));
  FillU32Kernel<<<592, 256, 0, stream>>>(reinterpret_cast<unsigned int*>(composite), (size_t)p.N * WH, flt_max_bits);
  cudaError_t err = cudaMemsetAsync(prior, 0, WH * sizeof(float), stream);
  if (err != cudaSuccess) return err;
  const dim3 block(32, 8);
  for (int i = 0; i < p.N; ++i) {
    if (!src_depth[i]) continue;
    const dim3 grid((gw + 31) / 32, (gh + 7) / 8);
    ProjectDepthKernel<<<grid, block, 0, stream>>>(src_depth[i], src_pitch[i], src_w[i], src_h[i],
                                                   p.poses + (size_t)i * SMVS_POSE_FLOATS, gw, gh, p.W, p.H, p.refK[0],
                                                   p.refK[1], p.refK[2], p.refK[3],
                                                   reinterpret_cast<unsigned int*>(composite) + (size_t)i * WH);
  }
  const dim3 grid((p.W + 31) / 32, (p.H + 7) / 8);
  CompositeDepthKernel<<<grid, block, 0, stream>>>(composite, p.N, p.W, p.H, p.depth, prior);
  CompositeNormalKernel<<<grid, block, 0, stream>>>(p.depth, p.W, p.H, p.refiK[0], p.refiK[1], p.refiK[2], p.refiK[3],
                                                    p.normal);
  return cudaGetLastError();
}

}  // namespace smvs
