// smvs_kernels.cu — per-pixel kernels (image conversion, reference moments,
// initialisation, mask, geometric-consistency filter) and the dispatch over
// the window-templated PatchMatch kernels of smvs_sweep.cuh.
#include <atomic>
#include <mutex>

#include <cuda_fp16.h>

#include "smvs_device.cuh"
#include "smvs_kernels.h"

namespace smvs {

namespace detail {
template <int R, int S>
cudaError_t LaunchWindow(const Batch& b, int op, int colour, cudaStream_t stream);
template <int R, int S>
cudaError_t ConfigureWindow();
}

namespace {

__device__ __forceinline__ float RefAt(const float* ref, int W, int H, int r, int c) {
  return (r >= 0 && r < H && c >= 0 && c < W) ? __ldg(ref + (size_t)r * W + c) : 0.0f;
}

// ---------------------------------------------------------------------------
// Image conversion: caller pixels (u8 / f32 grey 0..255) into device storage.
// normalise: values / 255 (u8 storage keeps the byte).
// ---------------------------------------------------------------------------
__global__ void ConvertImageKernel(const void* __restrict__ in, int in_format, size_t in_stride, int w, int h,
                                   void* __restrict__ out, int out_storage, size_t out_pitch) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const char* irow = (const char*)in + in_stride * y;
  const float g = (in_format == SMVS_PIX_U8) ? (float)((const uint8_t*)irow)[x] : ((const float*)irow)[x];
  char* orow = (char*)out + out_pitch * y;
  if (out_storage == SMVS_STORE_U8) {
    const float q = fminf(255.f, fmaxf(0.f, rintf(g)));
    ((uint8_t*)orow)[x] = (uint8_t)q;
  } else if (out_storage == SMVS_STORE_F16) {
    ((__half*)orow)[x] = __float2half_rn(g / 255.0f);
  } else if (out_storage == SMVS_STORE_F32) {
    ((float*)orow)[x] = g / 255.0f;
  } else {  // reference image: uint8-quantised, normalised fp32
    const float q = fminf(255.f, fmaxf(0.f, rintf(g)));
    ((float*)orow)[x] = q / 255.0f;
  }
}

// GpuMatRefImage::FilterKernel (gpu_mat_ref_image.cu:16-56) fused with
// ComputeGradientMap (kernel_functions.cu:1655-1675).
__global__ void PrepRefKernel(JobParams p, float* __restrict__ ref_sum, float* __restrict__ ref_sqsum,
                              float* __restrict__ grad) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const float center = RefAt(p.ref, p.W, p.H, row, col);
  float cs = 0.f, css = 0.f, ws = 0.f;
  for (int wr = -p.R; wr <= p.R; wr += p.S)
    for (int wc = -p.R; wc <= p.R; wc += p.S) {
      const float color = RefAt(p.ref, p.W, p.H, row + wr, col + wc);
      const float cd = center - color;
      const float w = __expf(-(float)(wr * wr + wc * wc) * p.sn - cd * cd * p.cn);
      cs += w * color;
      css += w * color * color;
      ws += w;
    }
  cs /= ws;
  css /= ws;
  const size_t pix = (size_t)row * p.W + col;
  ref_sum[pix] = cs;
  ref_sqsum[pix] = css;
  const float kx[3][3] = {{-3, 0, 3}, {-10, 0, 10}, {-3, 0, 3}};
  const float ky[3][3] = {{-3, -10, -3}, {0, 0, 0}, {3, 10, 3}};
  float gx = 0.f, gy = 0.f;
#pragma unroll
  for (int dr = -1; dr <= 1; ++dr)
#pragma unroll
    for (int dc = -1; dc <= 1; ++dc) {
      const float color = RefAt(p.ref, p.W, p.H, row + dr, col + dc);
      gx += color * kx[dr + 1][dc + 1];
      gy += color * ky[dr + 1][dc + 1];
    }
  grad[pix] = sqrtf(gx * gx + gy * gy);
}

// InitWorkspace: random branch (FillWithRandomNumbers, gpu_mat.h:114-130 +
// InitNormalMap, kernel_functions.cu:689-701) or given-map branch (InitDepthMap,
// kernel_functions.cu:703-737); also clears view_sel (patch_match_cuda.cu:677).
__global__ void InitKernel(JobParams p, int random_init, float dmin, float dmax) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const size_t WH = (size_t)p.W * p.H;
  const size_t pix = (size_t)row * p.W + col;
  Rng r(p.stage_key, (uint32_t)pix);
  const float vd[3] = {p.refiK[0] * col + p.refiK[1], p.refiK[2] * row + p.refiK[3], 1.0f};
  float d, n[3];
  if (random_init) {
    d = r.Uniform() * (dmax - dmin) + dmin;
    RandomNormal(r, vd, n);
  } else {
    d = p.depth[pix];
    n[0] = p.normal[pix]; n[1] = p.normal[WH + pix]; n[2] = p.normal[2 * WH + pix];
    if (d <= 0) {
      d = r.Uniform() * (dmax - dmin) + dmin;
      RandomNormal(r, vd, n);
    }
    if (Dot3(n, vd) >= 0) RandomNormal(r, vd, n);
  }
  p.depth[pix] = d;
  p.normal[pix] = n[0]; p.normal[WH + pix] = n[1]; p.normal[2 * WH + pix] = n[2];
  p.view_sel[pix] = 0u;
}


// ComputeCurvatureMap, kernel_functions.cu:1603-1653: slice 0 = Scharr gradient
// of the reference x 1e4 (clamped to 32767), slice 1 = median angle between
// the normal and its 5x5 neighbours x 1e4.
__global__ void CurvatureKernel(JobParams p, uint16_t* __restrict__ curv) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const size_t WH = (size_t)p.W * p.H;
  const size_t pix = (size_t)row * p.W + col;
  const float kx[3][3] = {{-3, 0, 3}, {-10, 0, 10}, {-3, 0, 3}};
  const float ky[3][3] = {{-3, -10, -3}, {0, 0, 0}, {3, 10, 3}};
  float gx = 0.f, gy = 0.f;
#pragma unroll
  for (int dr = -1; dr <= 1; ++dr)
#pragma unroll
    for (int dc = -1; dc <= 1; ++dc) {
      const float color = RefAt(p.ref, p.W, p.H, row + dr, col + dc);
      gx += color * kx[dr + 1][dc + 1];
      gy += color * ky[dr + 1][dc + 1];
    }
  const float grad = sqrtf(gx * gx + gy * gy);
  const int min_x = max(col - 2, 0), max_x = min(col + 2, p.W - 1);
  const int min_y = max(row - 2, 0), max_y = min(row + 2, p.H - 1);
  const float n0 = p.normal[pix], n1 = p.normal[WH + pix], n2 = p.normal[2 * WH + pix];
  float angles[24];
  int cnt = 0;
  for (int y = min_y; y <= max_y; ++y)
    for (int x = min_x; x <= max_x; ++x) {
      if (y == row && x == col) continue;
      const size_t q = (size_t)y * p.W + x;
      angles[cnt++] = acosf(n0 * p.normal[q] + n1 * p.normal[WH + q] + n2 * p.normal[2 * WH + q]);
    }
  curv[pix] = (uint16_t)fminf(grad * 10000.f, 32767.f);
  float med = 3.14159265358979323846f * 10000.0f;
  if (cnt > 0) {
    for (int i = 0; i < cnt - 1; ++i)  // BubbleSort, utils.h:190-209
      for (int j = 0; j < cnt - 1 - i; ++j)
        if (angles[j] > angles[j + 1]) { const float t = angles[j]; angles[j] = angles[j + 1]; angles[j + 1] = t; }
    med = angles[cnt / 2] * 10000.0f;
  }
  // Float to uint16 the way the hardware converts (NaN -> 0, saturating).
  curv[WH + pix] = (med != med) ? (uint16_t)0 : (uint16_t)fminf(fmaxf(med, 0.f), 65535.f);
}

// ComputeGeomGradientMap, kernel_functions.cu:3095-3120 (pixels without depth
// get 0; the reference leaves them unwritten).
__global__ void GeomGradientKernel(JobParams p, float* __restrict__ ggrad) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const size_t pix = (size_t)row * p.W + col;
  const float depth = p.depth[pix];
  if (depth <= 0) { ggrad[pix] = 0.f; return; }
  const float kx[3][3] = {{-3, 0, 3}, {-10, 0, 10}, {-3, 0, 3}};
  const float ky[3][3] = {{-3, -10, -3}, {0, 0, 0}, {3, 10, 3}};
  float gx = 0.f, gy = 0.f;
  for (int dr = -1; dr <= 1; ++dr)
    for (int dc = -1; dc <= 1; ++dc) {
      const int nr = row + dr, nc = col + dc;
      if (nr < 0 || nr >= p.H || nc < 0 || nc >= p.W) continue;
      const float diff = fabsf(p.depth[(size_t)nr * p.W + nc] - depth) / depth;
      gx += diff * kx[dr + 1][dc + 1];
      gy += diff * ky[dr + 1][dc + 1];
    }
  ggrad[pix] = sqrtf(gx * gx + gy * gy);
}

// MedianFilter via Black/RedPixelFilter, kernel_functions.cu:3122-3280: edge-aware
// median of depth and of each normal component over up to 17 taps.
__global__ void MedianFilterKernel(JobParams p, const float* __restrict__ ggrad, float diff_thres, int colour) {
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  const int col = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((row + colour) & 1);
  if (col >= p.W || row >= p.H) return;
  const int W = p.W, H = p.H;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  const float grad_thres = 1.4f * diff_thres;
  float depths[17], nx[17], ny[17], nz[17];
  const float grad = ggrad[pix];
  const float cdepth = p.depth[pix];
  const float inv_cdepth = 1.0f / cdepth;
  int index = 0;
  depths[index] = cdepth;
  nx[index] = p.normal[pix]; ny[index] = p.normal[WH + pix]; nz[index] = p.normal[2 * WH + pix];
  index++;
  auto take = [&](int nr, int nc) {
    const size_t q = (size_t)nr * W + nc;
    depths[index] = p.depth[q];
    const float diff = fabsf(depths[index] - cdepth) * inv_cdepth;
    if (grad < grad_thres || (grad >= grad_thres && diff < diff_thres)) {
      nx[index] = p.normal[q]; ny[index] = p.normal[WH + q]; nz[index] = p.normal[2 * WH + q];
      index++;
    }
  };
  for (int i = 0; i < 2; ++i) {
    const int o = 2 * i + 1;
    if (row - o >= 0) take(row - o, col);
    if (row + o < H) take(row + o, col);
    if (col - o >= 0) take(row, col - o);
    if (col + o < W) take(row, col + o);
  }
  const int dirs[8][2] = {{-2, 1}, {-1, 2}, {1, 2}, {2, 1}, {2, -1}, {1, -2}, {-1, -2}, {-2, -1}};
  for (int i = 0; i < 8; ++i) {
    const int nr = row + dirs[i][0], nc = col + dirs[i][1];
    if (nr >= 0 && nr < H && nc >= 0 && nc < W) take(nr, nc);
  }
  auto sort = [&](float* v) {
    for (int i = 0; i < index - 1; ++i)
      for (int j = 0; j < index - 1 - i; ++j)
        if (v[j] > v[j + 1]) { const float t = v[j]; v[j] = v[j + 1]; v[j + 1] = t; }
  };
  sort(depths); sort(nx); sort(ny); sort(nz);
  const int nth = index >> 1;
  const float inv_norm = rsqrtf(nx[nth] * nx[nth] + ny[nth] * ny[nth] + nz[nth] * nz[nth]);
  p.depth[pix] = depths[nth];
  p.normal[pix] = nx[nth] * inv_norm;
  p.normal[WH + pix] = ny[nth] * inv_norm;
  p.normal[2 * WH + pix] = nz[nth] * inv_norm;
}

// FilterDepthMap (confidence and planar-neighbour filter), kernel_functions.cu:
// 3282-3354, one checkerboard colour per launch. [quirk] the reference's grid
// covers rows r with r/2 < ceil((H/2)/16)*16, which skips the last row when H is
// odd and H/2 is a multiple of 16; the same rows are skipped here.
__global__ void ConfFilterKernel(JobParams p, float depth_thres, float conf_thres, int colour, int row_pairs) {
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  const int col = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((row + colour) & 1);
  if (col >= p.W || row >= p.H || (row >> 1) >= row_pairs) return;
  const int W = p.W, H = p.H;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  const float depth = p.depth[pix];
  if (depth <= 0) return;
  const float n[3] = {p.normal[pix], p.normal[WH + pix], p.normal[2 * WH + pix]};
  const float conf = p.conf[pix];
  const float* iK = p.refiK;
  const float pt[3] = {depth * (iK[0] * col + iK[1]), depth * (iK[2] * row + iK[3]), depth};
  int good = 0;
  for (int i = 0; i < 4; ++i) {
    const int u = col + (i == 0 ? -1 : (i == 2 ? 1 : 0)), v = row + (i == 1 ? -1 : (i == 3 ? 1 : 0));
    if (u < 0 || u >= W || v < 0 || v >= H) continue;
    const size_t q = (size_t)v * W + u;
    const float nd = p.depth[q];
    const float nn[3] = {p.normal[q], p.normal[WH + q], p.normal[2 * WH + q]};
    const float nconf = p.conf[q];
    const float np[3] = {nd * (iK[0] * u + iK[1]), nd * (iK[2] * v + iK[3]), nd};
    const float d1 = fabsf((pt[0] - np[0]) * n[0] + (pt[1] - np[1]) * n[1] + (pt[2] - np[2]) * n[2]);
    const float d2 = fabsf((pt[0] - np[0]) * nn[0] + (pt[1] - np[1]) * nn[1] + (pt[2] - np[2]) * nn[2]);
    if ((conf < conf_thres && d1 / depth < depth_thres) || (nconf < conf_thres && d2 / nd < depth_thres)) good++;
  }
  if (good < 2) {
    p.depth[pix] = 0.f;
    p.normal[pix] = 0.f; p.normal[WH + pix] = 0.f; p.normal[2 * WH + pix] = 0.f;
    p.conf[pix] = 0.f;
  }
}

// MaskDepthMapKernel, kernel_functions.cu:3080-3093 ([quirk] last row and
// column are left untouched).
__global__ void MaskKernel(JobParams p, const uint8_t* __restrict__ mask) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (row >= p.H - 1 || col >= p.W - 1) return;
  const size_t pix = (size_t)row * p.W + col;
  if (mask[pix] == 0) p.depth[pix] = 0.0f;
}

// FilterDepthMapsKernel (kernel_functions.cu:3356-3410) and
// DeduplicDepthMapsKernel (:3452-3487).
__global__ void FilterDepthMapsKernel(JobParams p, const float* __restrict__ in_depth, float* __restrict__ out_depth,
                                      int min_consistent, float filter_max_cost, int dedup) {
  __shared__ float poses[SMVS_MAX_SRC * SMVS_POSE_FLOATS];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = tid; i < p.N * SMVS_POSE_FLOATS; i += blockDim.x * blockDim.y) poses[i] = p.poses[i];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const size_t pix = (size_t)row * p.W + col;
  const float d = in_depth[pix];
  if (d < 1e-6f) { out_depth[pix] = 0.0f; return; }
  const float np[3] = {p.refiK[0] * col + p.refiK[1], p.refiK[2] * row + p.refiK[3], 1.0f};
  int good = 0;
  for (int v = 0; v < p.N; ++v) {
    const bool ok = GeomCost(poses + v * SMVS_POSE_FLOATS, p.dep_tex[v], (float)row, (float)col, d, np, p.refK,
                             p.geom_max) <= filter_max_cost;
    if (ok && dedup) { out_depth[pix] = 0.0f; return; }
    good += ok;
  }
  out_depth[pix] = (!dedup && good < min_consistent) ? 0.0f : d;
}


// Dispatch over the window sizes the reference supports
// (kernel_functions.cu:1343-1400).
cudaError_t LaunchWindowOp(const Batch& b, int op, int colour, cudaStream_t stream) {
  const int R = b.R, S = b.S;
  if (R == 5 && S == 1) return detail::LaunchWindow<5, 1>(b, op, colour, stream);
  if (R == 3 && S == 1) return detail::LaunchWindow<3, 1>(b, op, colour, stream);
  if (R == 7 && S == 1) return detail::LaunchWindow<7, 1>(b, op, colour, stream);
  if (R == 3 && S == 2) return detail::LaunchWindow<3, 2>(b, op, colour, stream);
  if (R == 4 && S == 2) return detail::LaunchWindow<4, 2>(b, op, colour, stream);
  if (R == 5 && S == 2) return detail::LaunchWindow<5, 2>(b, op, colour, stream);
  if (R == 7 && S == 2) return detail::LaunchWindow<7, 2>(b, op, colour, stream);
  return cudaErrorInvalidValue;
}

__global__ void AdvanceKernel(int* __restrict__ iters, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) iters[i] += 1;
}

}  // namespace

bool SupportedWindow(int R, int S) {
  return (S == 1 && (R == 3 || R == 5 || R == 7)) || (S == 2 && (R == 3 || R == 4 || R == 5 || R == 7));
}

cudaError_t LaunchConvertImage(const void* in, int in_format, size_t in_stride, int w, int h, void* out,
                               int out_storage, size_t out_pitch, int /*normalise*/, cudaStream_t stream) {
  dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
  ConvertImageKernel<<<grid, block, 0, stream>>>(in, in_format, in_stride, w, h, out, out_storage, out_pitch);
  return cudaGetLastError();
}

cudaError_t LaunchPrepRef(const JobParams& p, float* ref_sum, float* ref_sqsum, float* grad, cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  PrepRefKernel<<<grid, block, 0, stream>>>(p, ref_sum, ref_sqsum, grad);
  return cudaGetLastError();
}

cudaError_t LaunchInit(const JobParams& p, int random_init, float opt_dmin, float opt_dmax, cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  InitKernel<<<grid, block, 0, stream>>>(p, random_init, opt_dmin, opt_dmax);
  return cudaGetLastError();
}

cudaError_t LaunchInitConf(const Batch& b, cudaStream_t stream) { return LaunchWindowOp(b, 0, 0, stream); }

cudaError_t LaunchSweep(const Batch& b, int colour, cudaStream_t stream) {
  return LaunchWindowOp(b, 1, colour, stream);
}

cudaError_t LaunchLocalOpt(const Batch& b, int colour, cudaStream_t stream) {
  return LaunchWindowOp(b, 2, colour, stream);
}

cudaError_t LaunchAdvance(int* iters, int num_jobs, cudaStream_t stream) {
  if (num_jobs <= 0) return cudaSuccess;
  AdvanceKernel<<<(num_jobs + 127) / 128, 128, 0, stream>>>(iters, num_jobs);
  return cudaGetLastError();
}

int ViewBucket(int N) { return (N + 3) & ~3; }

static std::atomic<int> g_persistent_grid_cap{0};
int PersistentGridCap() { return g_persistent_grid_cap.load(std::memory_order_relaxed); }
void SetPersistentGridCap(int max_blocks) { g_persistent_grid_cap.store(max_blocks, std::memory_order_relaxed); }

int FitThreadsPerPixel(int R, int nb, int bx, int tpp) {
  for (int t = tpp; t <= 4; t *= 2)
    if (ValidSweepShape(bx, t) && SweepKernelSmem(R, nb, bx, t) <= kMaxDynamicSmem &&
        LocalKernelSmem(R, nb, bx, t) <= kMaxDynamicSmem)
      return t;
  return 0;
}

cudaError_t ConfigureKernels() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return cudaSuccess;
  if (e == cudaSuccess) e = detail::ConfigureWindow<5, 1>();
  if (e == cudaSuccess) e = detail::ConfigureWindow<3, 1>();
  if (e == cudaSuccess) e = detail::ConfigureWindow<7, 1>();
  if (e == cudaSuccess) e = detail::ConfigureWindow<3, 2>();
  if (e == cudaSuccess) e = detail::ConfigureWindow<4, 2>();
  if (e == cudaSuccess) e = detail::ConfigureWindow<5, 2>();
  if (e == cudaSuccess) e = detail::ConfigureWindow<7, 2>();
  if (e == cudaSuccess) done[dev] = true;
  return e;
}

cudaError_t LaunchCurvature(const JobParams& p, uint16_t* curv, cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  CurvatureKernel<<<grid, block, 0, stream>>>(p, curv);
  return cudaGetLastError();
}

cudaError_t LaunchGeomGradient(const JobParams& p, float* ggrad, cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  GeomGradientKernel<<<grid, block, 0, stream>>>(p, ggrad);
  return cudaGetLastError();
}

cudaError_t LaunchMedianFilter(const JobParams& p, const float* ggrad, float diff_thres, int colour,
                               cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 63) / 64, (p.H + 7) / 8);
  MedianFilterKernel<<<grid, block, 0, stream>>>(p, ggrad, diff_thres, colour);
  return cudaGetLastError();
}

cudaError_t LaunchConfFilter(const JobParams& p, float depth_thres, float conf_thres, int colour,
                             cudaStream_t stream) {
  const int row_pairs = ((p.H / 2) + 15) / 16 * 16;  // the reference's grid, patch_match_cuda.cu:1018-1037
  dim3 block(32, 8), grid((p.W + 63) / 64, (p.H + 7) / 8);
  ConfFilterKernel<<<grid, block, 0, stream>>>(p, depth_thres, conf_thres, colour, row_pairs);
  return cudaGetLastError();
}

cudaError_t LaunchMask(const JobParams& p, const uint8_t* mask, cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  MaskKernel<<<grid, block, 0, stream>>>(p, mask);
  return cudaGetLastError();
}

cudaError_t LaunchFilterDepthMaps(const JobParams& p, const float* in_depth, float* out_depth, int min_consistent,
                                  float filter_max_cost, int dedup, cudaStream_t stream) {
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  FilterDepthMapsKernel<<<grid, block, 0, stream>>>(p, in_depth, out_depth, min_consistent, filter_max_cost, dedup);
  return cudaGetLastError();
}

}  // namespace smvs
