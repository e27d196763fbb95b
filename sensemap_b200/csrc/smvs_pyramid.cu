// smvs_pyramid.cu — the coarse-to-fine image pyramid on the GPU.
//
// The reference runs its PatchMatch passes per pyramid level on images it
// rescales on the host (PatchMatchController::ProcessProblem,
// patch_match_controller.cc:4407-4410 and 4610, Image::Rescale,
// src/mvs/image.cc:44-70, through FreeImage's bilinear filter), and carries
// depth and normal maps between levels by DepthMap::Rescale / NormalMap::
// Rescale (src/mvs/depth_map.cc:32-55, src/mvs/normal_map.cc:27-72), i.e.
// InterpolateImage -> ResampleImageBilinear (src/util/mat.cc:18-58, 129-137)
// followed by a re-normalisation of the normals. This unit does both on the
// device:
// * RescaleImageKernel: separable resampling with the bilinear (triangle)
//   filter widened by the inverse scale when minifying (the published
//   algorithm of FreeImage's FILTER_BILINEAR rescale; FreeImage itself is a
//   third-party library that is not part of the reference tree), weights
//   normalised over the pixels inside the image, result rounded to an
//   integer grey level 0..255 like the 8-bit bitmap.
// * ResampleMapKernel: ResampleImageBilinear exactly (same float expressions,
//   constant-0 border), for the depth map and each normal slice, then the
//   normal re-normalisation. This unit is compiled without FMA contraction
//   and with IEEE division and square root, so its results equal the C
//   restatement in the oracle bit for bit.
#include <cmath>

#include <cuda_runtime.h>

#include "../../include/smvs.h"

extern "C" void smvs_internal_set_error(const char* msg);

namespace {

// One pass of the separable image filter over rows (axis 0 = along x).
// out[y][x] = sum_i w_i in[y][i] / sum_i w_i for the input pixels i whose
// centres lie within the filter support around the output pixel's centre.
__global__ void ResampleRowsKernel(const float* __restrict__ in, int w, int h, float* __restrict__ out, int ow,
                                   float scale) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= ow || y >= h) return;
  const float support = scale < 1.0f ? 1.0f / scale : 1.0f;  // triangle half-width in input pixels
  const float fscale = scale < 1.0f ? scale : 1.0f;
  const float c = ((float)x + 0.5f) / scale;
  int i0 = (int)floorf(c - support), i1 = (int)ceilf(c + support);
  i0 = i0 < 0 ? 0 : i0;
  i1 = i1 > w - 1 ? w - 1 : i1;
  float acc = 0.f, wsum = 0.f;
  const float* row = in + (size_t)y * w;
  for (int i = i0; i <= i1; ++i) {
    const float wt = 1.0f - fabsf(((float)i + 0.5f) - c) * fscale;
    if (wt <= 0.f) continue;
    acc += wt * row[i];
    wsum += wt;
  }
  out[(size_t)y * ow + x] = wsum > 0.f ? acc / wsum : 0.f;
}

// The same filter along y; rounds to an integer grey level.
__global__ void ResampleColsKernel(const float* __restrict__ in, int w, int h, float* __restrict__ out, int oh,
                                   float scale) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= oh) return;
  const float support = scale < 1.0f ? 1.0f / scale : 1.0f;
  const float fscale = scale < 1.0f ? scale : 1.0f;
  const float c = ((float)y + 0.5f) / scale;
  int i0 = (int)floorf(c - support), i1 = (int)ceilf(c + support);
  i0 = i0 < 0 ? 0 : i0;
  i1 = i1 > h - 1 ? h - 1 : i1;
  float acc = 0.f, wsum = 0.f;
  for (int i = i0; i <= i1; ++i) {
    const float wt = 1.0f - fabsf(((float)i + 0.5f) - c) * fscale;
    if (wt <= 0.f) continue;
    acc += wt * in[(size_t)i * w + x];
    wsum += wt;
  }
  const float v = wsum > 0.f ? acc / wsum : 0.f;
  out[(size_t)y * w + x] = fminf(255.f, fmaxf(0.f, rintf(v)));
}

__device__ __forceinline__ float PixelOr0(const float* d, int rows, int cols, int r, int c) {
  return (r >= 0 && c >= 0 && r < rows && c < cols) ? d[(size_t)r * cols + c] : 0.0f;
}

// ResampleImageBilinear (mat.cc:18-58) of `planes` planes, then (normals) the
// re-normalisation of NormalMap::Rescale (normal_map.cc:57-72).
__global__ void ResampleMapKernel(const float* __restrict__ in, int rows, int cols, float* __restrict__ out,
                                  int new_rows, int new_cols, int planes, int renormalise) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= new_cols || r >= new_rows) return;
  const float scale_r = (float)rows / (float)new_rows;
  const float scale_c = (float)cols / (float)new_cols;
  const float r_i = ((float)r + 0.5f) * scale_r - 0.5f;
  const int r_i_min = (int)floorf(r_i);
  const int r_i_max = r_i_min + 1;
  const float d_r_min = r_i - (float)r_i_min;
  const float d_r_max = (float)r_i_max - r_i;
  const float c_i = ((float)c + 0.5f) * scale_c - 0.5f;
  const int c_i_min = (int)floorf(c_i);
  const int c_i_max = c_i_min + 1;
  const float d_c_min = c_i - (float)c_i_min;
  const float d_c_max = (float)c_i_max - c_i;
  const size_t in_plane = (size_t)rows * cols, out_plane = (size_t)new_rows * new_cols;
  const size_t o = (size_t)r * new_cols + c;
  float v[3];
  for (int p = 0; p < planes; ++p) {
    const float* d = in + p * in_plane;
    const float value1 = d_c_max * PixelOr0(d, rows, cols, r_i_min, c_i_min) +
                         d_c_min * PixelOr0(d, rows, cols, r_i_min, c_i_max);
    const float value2 = d_c_max * PixelOr0(d, rows, cols, r_i_max, c_i_min) +
                         d_c_min * PixelOr0(d, rows, cols, r_i_max, c_i_max);
    v[p] = d_r_max * value1 + d_r_min * value2;
  }
  if (renormalise && planes == 3) {
    const float sq = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
    if (sq > 0.f) {
      const float n = sqrtf(sq);
      v[0] = v[0] / n; v[1] = v[1] / n; v[2] = v[2] / n;
    }
  }
  for (int p = 0; p < planes; ++p) out[p * out_plane + o] = v[p];
}

int Fail(int code, const char* msg) {
  smvs_internal_set_error(msg);
  return code;
}

}  // namespace

extern "C" {

int smvs_pyramid_level_size(int width, int height, int level, int* out_width, int* out_height, float* factor) {
  if (width <= 0 || height <= 0 || level < 0 || !out_width || !out_height)
    return Fail(SMVS_EINVAL, "smvs_pyramid_level_size: bad arguments");
  // patch_match_controller.cc:4407-4410: 1 / 2^level, but never below 320
  // pixels on the longer side; image.cc:51-52: rounded sizes.
  float f = 1.0f / std::pow(2.0f, (float)level);
  const float max_size = (float)(width > height ? width : height);
  const float min_size = std::min(320.f, max_size);
  f = std::max(f, min_size / max_size);
  *out_width = (int)std::round(width * f);
  *out_height = (int)std::round(height * f);
  if (factor) *factor = f;
  return SMVS_OK;
}

int smvs_rescale_image(const float* in, int width, int height, float* out, int out_width, int out_height,
                       void* scratch, void* stream) {
  if (!in || !out || !scratch || width <= 0 || height <= 0 || out_width <= 0 || out_height <= 0)
    return Fail(SMVS_EINVAL, "smvs_rescale_image: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  float* tmp = static_cast<float*>(scratch);  // out_width x height
  dim3 blk(32, 8);
  ResampleRowsKernel<<<dim3((out_width + 31) / 32, (height + 7) / 8), blk, 0, s>>>(
      in, width, height, tmp, out_width, (float)out_width / (float)width);
  ResampleColsKernel<<<dim3((out_width + 31) / 32, (out_height + 7) / 8), blk, 0, s>>>(
      tmp, out_width, height, out, out_height, (float)out_height / (float)height);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return Fail(SMVS_ECUDA, cudaGetErrorString(e));
  return SMVS_OK;
}

int smvs_resample_maps(const float* depth, const float* normal, int width, int height, float* out_depth,
                       float* out_normal, int out_width, int out_height, void* stream) {
  if ((!depth && !normal) || (depth && !out_depth) || (normal && !out_normal) || width <= 0 || height <= 0 ||
      out_width <= 0 || out_height <= 0)
    return Fail(SMVS_EINVAL, "smvs_resample_maps: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  dim3 blk(32, 8), grd((out_width + 31) / 32, (out_height + 7) / 8);
  if (depth) ResampleMapKernel<<<grd, blk, 0, s>>>(depth, height, width, out_depth, out_height, out_width, 1, 0);
  if (normal) ResampleMapKernel<<<grd, blk, 0, s>>>(normal, height, width, out_normal, out_height, out_width, 3, 1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return Fail(SMVS_ECUDA, cudaGetErrorString(e));
  return SMVS_OK;
}

}  // extern "C"
