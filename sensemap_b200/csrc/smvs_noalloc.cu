// smvs_noalloc.cu — geometric-consistency filter that allocates nothing.
//
// For callers that cannot call cudaMalloc: a serving process that reserved its
// whole device-memory budget at start-up and may not grow it per request, or
// host code called back from a framework that owns every device allocation
// and forbids allocating behind its back. The caller passes device buffers for
// every input and output; the kernel's scratch (the pose records of the source
// views) lives in a file-scope __device__ array that every GPU loading this
// library holds until the process exits. The records reach that array through
// a one-block kernel that takes them as a by-value kernel parameter, so no host
// buffer has to outlive the call.
//
// Same arithmetic as smvs_run_filter (FilterDepthMapsKernel,
// kernel_functions.cu:3356-3487), except that source depth maps are read from
// the caller's dense buffers with the bilinear weights the texture unit uses
// (8-bit positions, integer 1/256 weights with w11 = round(A*B/256)) instead
// of through texture objects, which this entry point may not create.
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/smvs.h"
#include "smvs_device.cuh"

extern "C" void smvs_internal_set_error(const char* msg);

// Scratch: one 43-float pose record per source view (5,504 bytes). Every call
// overwrites the records it uses before its filter kernel reads them.
static __device__ __align__(256) float g_filter_scratch[SMVS_NOALLOC_MAX_SRC * SMVS_POSE_FLOATS];

namespace {

// The pose records of one call, passed by value to the kernel that stores them
// in the scratch array (5,504 bytes, within the 32 KB kernel-parameter limit
// of CUDA 12.1+ on sm_70 and later).
struct PoseRecords {
  float v[SMVS_NOALLOC_MAX_SRC * SMVS_POSE_FLOATS];
};

__global__ void StorePoseRecordsKernel(const PoseRecords rec, int count, float* __restrict__ scratch) {
  for (int i = threadIdx.x; i < count; i += blockDim.x) scratch[i] = rec.v[i];
}

struct NoAllocParams {
  int W, H, N;
  float refK[4], refiK[4];
  float geom_max, filter_max_cost;
  int min_consistent, dedup;
  const float* ref_depth;
  float* out_depth;
  const float* src_depth[SMVS_NOALLOC_MAX_SRC];
  int src_w[SMVS_NOALLOC_MAX_SRC], src_h[SMVS_NOALLOC_MAX_SRC];
};

__device__ __forceinline__ float SampleBilinear(const float* __restrict__ img, int w, int h, float x, float y) {
  if (!(fabsf(x) < 1.0e7f && fabsf(y) < 1.0e7f)) return 0.0f;
  const float xb = x - 0.5f, yb = y - 0.5f;
  const float fx = floorf(xb), fy = floorf(yb);
  const int i = (int)fx, j = (int)fy;
  const int A = (int)floorf((xb - fx) * 256.0f + 0.5f);
  const int B = (int)floorf((yb - fy) * 256.0f + 0.5f);
  const int w11 = (A * B + 128) >> 8, w10 = A - w11, w01 = B - w11, w00 = 256 - A - B + w11;
  const bool i0 = i >= 0 && i < w, i1 = i + 1 >= 0 && i + 1 < w;
  const bool j0 = j >= 0 && j < h, j1 = j + 1 >= 0 && j + 1 < h;
  const float t00 = (i0 && j0) ? __ldg(img + (size_t)j * w + i) : 0.0f;
  const float t10 = (i1 && j0) ? __ldg(img + (size_t)j * w + i + 1) : 0.0f;
  const float t01 = (i0 && j1) ? __ldg(img + (size_t)(j + 1) * w + i) : 0.0f;
  const float t11 = (i1 && j1) ? __ldg(img + (size_t)(j + 1) * w + i + 1) : 0.0f;
  return ((float)w00 * t00 + (float)w10 * t10 + (float)w01 * t01 + (float)w11 * t11) * (1.0f / 256.0f);
}

// ComputeGeomConsistencyCost (kernel_functions.cu:570-633) with the source
// depth read from a dense buffer.
__device__ __forceinline__ float GeomCostDense(const float* pose, const float* depth_map, int w, int h, float row,
                                               float col, float depth, const float np[3], const float K[4],
                                               float max_cost) {
  const float* P = pose + 19;
  const float* iP = pose + 31;
  const float X0 = depth * np[0], X1 = depth * np[1], X2 = depth * np[2];
  const float ifz = 1.0f / (P[8] * X0 + P[9] * X1 + P[10] * X2 + P[11]);
  float scol = ifz * (P[0] * X0 + P[1] * X1 + P[2] * X2 + P[3]);
  float srow = ifz * (P[4] * X0 + P[5] * X1 + P[6] * X2 + P[7]);
  const float sd = SampleBilinear(depth_map, w, h, scol + 0.5f, srow + 0.5f);
  if (sd == 0.0f) return max_cost;
  scol *= sd;
  srow *= sd;
  const float bx = iP[0] * scol + iP[1] * srow + iP[2] * sd + iP[3];
  const float by = iP[4] * scol + iP[5] * srow + iP[6] * sd + iP[7];
  const float bz = iP[8] * scol + iP[9] * srow + iP[10] * sd + iP[11];
  const float ibz = 1.0f / bz;
  const float bcol = ibz * K[0] * bx + K[1];
  const float brow = ibz * K[2] * by + K[3];
  const float dc = col - bcol, dr = row - brow;
  return fminf(max_cost, sqrtf(dc * dc + dr * dr));
}

__global__ void FilterDepthMapsNoAllocKernel(NoAllocParams p, const float* __restrict__ scratch_poses) {
  __shared__ float poses[SMVS_NOALLOC_MAX_SRC * SMVS_POSE_FLOATS];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = tid; i < p.N * SMVS_POSE_FLOATS; i += blockDim.x * blockDim.y) poses[i] = scratch_poses[i];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const size_t pix = (size_t)row * p.W + col;
  const float d = p.ref_depth[pix];
  if (d < 1e-6f) { p.out_depth[pix] = 0.0f; return; }
  const float np[3] = {p.refiK[0] * col + p.refiK[1], p.refiK[2] * row + p.refiK[3], 1.0f};
  int good = 0;
  for (int v = 0; v < p.N; ++v) {
    const bool ok = GeomCostDense(poses + v * SMVS_POSE_FLOATS, p.src_depth[v], p.src_w[v], p.src_h[v], (float)row,
                                  (float)col, d, np, p.refK, p.geom_max) <= p.filter_max_cost;
    if (ok && p.dedup) { p.out_depth[pix] = 0.0f; return; }
    good += ok;
  }
  p.out_depth[pix] = (!p.dedup && good < p.min_consistent) ? 0.0f : d;
}

// Device address of the scratch array, looked up once per device.
std::mutex g_scratch_mutex;
float* g_scratch_ptr[64] = {nullptr};

int Fail(int code, const char* msg) {
  smvs_internal_set_error(msg);
  return code;
}

}  // namespace

// Defined in smvs_engine.cu: the 43-float pose record of a source view.
void smvs_internal_pose_record(const smvs_view* ref, const smvs_view* src, float* out43);

extern "C" int smvs_filter_depth_map_noalloc(const smvs_options* opt, const smvs_problem* prob, float* out_depth,
                                             int deduplication, void* stream) {
  if (!opt || !prob || !out_depth) return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: null argument");
  // The options pass the same check as smvs_create's (which smvs_run_filter
  // goes through), so both entry points reject the same option sets.
  const int ost = smvs_options_check(opt);
  if (ost != SMVS_OK) return ost;
  if (prob->memory != SMVS_MEM_DEVICE)
    return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: depth maps must be device buffers (SMVS_MEM_DEVICE)");
  if (prob->num_src < 1 || prob->num_src > SMVS_NOALLOC_MAX_SRC)
    return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: num_src must be 1..SMVS_NOALLOC_MAX_SRC (32)");
  if (!prob->ref.depth || prob->ref.width <= 0 || prob->ref.height <= 0)
    return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: the reference view needs width, height and depth");
  if (prob->ref.K[0] == 0.f || prob->ref.K[4] == 0.f)
    return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: zero focal length");
  if (!prob->src) return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: null source view list");
  for (int i = 0; i < prob->num_src; ++i) {
    if (!prob->src[i].depth || prob->src[i].width <= 0 || prob->src[i].height <= 0)
      return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: every source view needs width, height and depth");
    if (prob->src[i].K[0] == 0.f || prob->src[i].K[4] == 0.f)
      return Fail(SMVS_EINVAL, "smvs_filter_depth_map_noalloc: zero focal length in a source view");
  }

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return Fail(SMVS_ECUDA, "smvs_filter_depth_map_noalloc: no current CUDA device");
  float* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
      void* ptr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&ptr, g_filter_scratch);
      if (e != cudaSuccess) return Fail(SMVS_ECUDA, cudaGetErrorString(e));
      g_scratch_ptr[dev] = (float*)ptr;
    }
    scratch = g_scratch_ptr[dev];
  }

  NoAllocParams p;
  memset(&p, 0, sizeof(p));
  p.W = prob->ref.width;
  p.H = prob->ref.height;
  p.N = prob->num_src;
  const float* K = prob->ref.K;
  p.refK[0] = K[0]; p.refK[1] = K[2]; p.refK[2] = K[4]; p.refK[3] = K[5];
  p.refiK[0] = 1.0f / p.refK[0];
  p.refiK[1] = -p.refK[1] / p.refK[0];
  p.refiK[2] = 1.0f / p.refK[2];
  p.refiK[3] = -p.refK[3] / p.refK[2];
  p.geom_max = (float)opt->geom_consistency_max_cost;
  p.filter_max_cost = (float)opt->filter_geom_consistency_max_cost;
  p.min_consistent = opt->filter_min_num_consistent < p.N ? opt->filter_min_num_consistent : p.N;
  p.dedup = deduplication ? 1 : 0;
  p.ref_depth = prob->ref.depth;
  p.out_depth = out_depth;
  PoseRecords rec;
  memset(&rec, 0, sizeof(rec));
  for (int i = 0; i < p.N; ++i) {
    p.src_depth[i] = prob->src[i].depth;
    p.src_w[i] = prob->src[i].width;
    p.src_h[i] = prob->src[i].height;
    smvs_internal_pose_record(&prob->ref, &prob->src[i], rec.v + i * SMVS_POSE_FLOATS);
  }
  // An error left pending on this thread by earlier CUDA work would otherwise
  // surface as this call's launch error; report it (this reads and clears it)
  // and enqueue nothing.
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "smvs_filter_depth_map_noalloc: a CUDA error from earlier work was pending on this thread (%s); "
             "nothing was enqueued",
             cudaGetErrorName(e));
    return Fail(SMVS_ECUDA, msg);
  }
  cudaStream_t s = (cudaStream_t)stream;
  // The records of this call replace the previous call's (stream-ordered
  // before the filter kernel that reads them).
  StorePoseRecordsKernel<<<1, 256, 0, s>>>(rec, p.N * SMVS_POSE_FLOATS, scratch);
  dim3 block(32, 8), grid((p.W + 31) / 32, (p.H + 7) / 8);
  FilterDepthMapsNoAllocKernel<<<grid, block, 0, s>>>(p, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return Fail(SMVS_ECUDA, cudaGetErrorString(e));
  return SMVS_OK;
}
