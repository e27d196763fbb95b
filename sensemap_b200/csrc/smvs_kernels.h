// smvs_kernels.h — host-side launchers of the PatchMatch kernels (internal).
#pragma once

#include <cstdint>
#include <cuda.h>  // CUtensorMap (type only; the encoder is reached through the runtime)
#include <cuda_runtime.h>

#include "../../include/smvs.h"

namespace smvs {

constexpr int kMaxIterations = 32;  // th_mc table size (num_iterations limit)

// Per-job parameter block. It replaces the reference's __constant__
// ref_K/ref_inv_K slots (kernel_functions.cu:18-20) and its SweepOptions
// struct (kernel_functions.h:67-111). Per-pixel kernels take it by value; the
// batched checkerboard kernels read an array of them from device memory (one
// entry per job of a batch) and stage their job's entry in shared memory.
struct alignas(16) JobParams {
  int W, H, N, R, S;
  float sn, cn;                     // BilateralWeightComputer normalisations (utils.h:72-92)
  float depth_min, depth_max;       // options' depth range (float)
  float rand_depth_ratio, rand_a1, rand_a2;
  float th_mc, max_mc, inv_beta2;   // th_mc: per-launch value of the per-pixel kernels
  int num_samples, num_good, num_bad, random_opt, geom, thk;
  float geom_reg, geom_max;
  float refK[4], refiK[4];
  uint64_t stage_key;               // per-launch RNG stage key of the per-pixel kernels
  uint64_t seed;                    // job seed (batched kernels derive stage keys from it)
  int block_x;                      // checkerboard kernels: threads per block in x (256 / block_x in y)
  int num_iterations;
  int local_opt;
  int blocks_x;                     // batched launches: this job's checkerboard blocks per row
  int conf_blocks_x;                // batched InitConf launches: blocks per row
  int tma_box_w, tma_box_h;         // box of this job's reference tensor map; 0 = stage with loads
  float th_tab[kMaxIterations];     // th_mc of each iteration (patch_match_cuda.cu:778-779)
  // State maps (dense row-major; normal and cost planar).
  float* depth;
  float* normal;
  float* conf;
  float* cost;
  uint32_t* view_sel;
  // Reference-view data.
  const float* ref;        // W*H, [0,1]
  const float* ref_sum;    // W*H
  const float* ref_sqsum;  // W*H
  const float* grad;       // W*H
  const float* poses;      // N*43
  cudaTextureObject_t src_tex[SMVS_MAX_SRC];
  cudaTextureObject_t dep_tex[SMVS_MAX_SRC];
};

// A batch of jobs for the checkerboard kernels: device arrays of job params,
// per-job iteration counters and block prefix sums (block_start[j] = first
// block of job j; block_start[num_jobs] = total blocks).
struct Batch {
  const JobParams* jobs;
  const int* iters;
  const int* block_start;       // checkerboard tiling (Sweep / LocalOpt)
  const int* conf_block_start;  // full tiling (InitConf)
  int num_jobs;
  int total_blocks;             // checkerboard tiling
  int total_conf_blocks;        // full tiling
  int block_x;                  // shared launch shape of the batch
  int R, S, NB;                 // shared window and view bucket of the batch
  const CUtensorMap* ref_maps;  // per job: reference image for TMA tile loads (jobs with tma_box_w > 0)
  int* status;                  // set to 1 when a bounded wait of a kernel gave up
};

// Reference tile of the checkerboard kernels (block bx x 256/bx threads, two
// columns per thread): rows [row0 - R, row0 + by + R), columns starting at
// col0 - R - RefTileShift(R), so that the first column is a multiple of 4
// floats (col0 is a multiple of 2 bx >= 16): a TMA box may only start on a
// 16-byte boundary. The tile's row stride is RefTileW.
__host__ __device__ inline int RefTileShift(int R) { return (4 - (R & 3)) & 3; }
__host__ __device__ inline int RefTileW(int bx, int R) { return (2 * bx + 2 * R + RefTileShift(R) + 3) & ~3; }
__host__ __device__ inline int RefTileH(int bx, int R) { return 256 / bx + 2 * R; }

// Encodes the TMA descriptor of a dense W x H FP32 reference image for the
// checkerboard tile of launch shape bx and window R. Returns false (use plain
// loads) when the image rows are not a multiple of 16 bytes, the image is
// smaller than the box, or the driver does not provide the encoder.
bool EncodeRefMap(CUtensorMap* map, const float* ref, int W, int H, int bx, int R);

// All launchers enqueue on `stream` and return the launch status.
cudaError_t LaunchConvertImage(const void* in, int in_format, size_t in_stride, int w, int h, void* out,
                               int out_storage, size_t out_pitch, int normalise, cudaStream_t stream);
cudaError_t LaunchPrepRef(const JobParams& p, float* ref_sum, float* ref_sqsum, float* grad, cudaStream_t stream);
cudaError_t LaunchInit(const JobParams& p, int random_init, float opt_dmin, float opt_dmax, cudaStream_t stream);
// Batched checkerboard kernels: every job of `b` in one launch.
cudaError_t LaunchInitConf(const Batch& b, cudaStream_t stream);
cudaError_t LaunchSweep(const Batch& b, int colour, cudaStream_t stream);
cudaError_t LaunchLocalOpt(const Batch& b, int colour, cudaStream_t stream);
// iters[j] += 1 for every job of the batch (after both colours of an iteration).
cudaError_t LaunchAdvance(int* iters, int num_jobs, cudaStream_t stream);
// View bucket (max views of the M matrix) for N source views.
int ViewBucket(int N);
cudaError_t LaunchMask(const JobParams& p, const uint8_t* mask, cudaStream_t stream);
cudaError_t LaunchCurvature(const JobParams& p, uint16_t* curv, cudaStream_t stream);
cudaError_t LaunchGeomGradient(const JobParams& p, float* ggrad, cudaStream_t stream);
cudaError_t LaunchMedianFilter(const JobParams& p, const float* ggrad, float diff_thres, int colour, cudaStream_t stream);
cudaError_t LaunchConfFilter(const JobParams& p, float depth_thres, float conf_thres, int colour, cudaStream_t stream);
cudaError_t LaunchFilterDepthMaps(const JobParams& p, const float* in_depth, float* out_depth, int min_consistent,
                                  float filter_max_cost, int dedup, cudaStream_t stream);

bool SupportedWindow(int R, int S);

}  // namespace smvs
