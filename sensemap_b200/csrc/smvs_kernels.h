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
  int block_x;                      // checkerboard kernels: pixels per block row (each spans 2 image columns)
  int tpp;                          // checkerboard kernels: threads per pixel (1, 2 or 4)
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
  // Prior maps of the sweep (SweepOptions::prior_depth_ncc / propagate_depth,
  // kernel_functions.h:109-110). prior_mode 0: none; 1: has_prior_depth (the
  // given depth and normal weight every cost, kernel_functions.cu:1470-1486);
  // 2: propagate_depth (the projected median depth; normals and weights read
  // as 0). A NULL normal or weight map reads as 0.
  int prior_mode;
  const float* prior_depth;   // W*H
  const float* prior_normal;  // 3*W*H planar
  const float* prior_wgt;     // W*H
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
  int block_x;                  // shared launch shape of the batch: pixels per block row
  int tpp;                      // and threads per pixel (a block is 256 threads, 256 / tpp pixels)
  int R, S, NB;                 // shared window; NB = views per pixel in shared memory (>= every job's N)
  const CUtensorMap* ref_maps;  // per job: reference image for TMA tile loads (jobs with tma_box_w > 0)
  int* status;                  // set to 1 when a bounded wait of a kernel gave up
  int tma_polls;                // mbarrier polls before a TMA tile wait gives up (0 = the default bound)
  int tma_skip_copy;            // test hook: arm the tile barrier but issue no copy (its waits run out)
  int persistent;               // tpp == 1: a persistent grid strides over the tiles (0: one block per tile)
  int grid_cap;                 // test hook: at most this many persistent blocks (0 = the resident count)
};

// Checkerboard blocks: 256 threads, tpp threads per pixel, bx pixels per
// block row (two image columns each) and SweepRows(bx, tpp) pixel rows.
__host__ __device__ inline int SweepRows(int bx, int tpp) { return 256 / (tpp * bx); }
// Reference tile of a checkerboard block: rows [row0 - R, row0 + rows + R),
// columns starting at col0 - R - RefTileShift(R), so that the first column is
// a multiple of 4 floats (col0 is a multiple of 2 bx >= 16): a TMA box may only
// start on a 16-byte boundary. The tile's row stride is RefTileW.
__host__ __device__ inline int RefTileShift(int R) { return (4 - (R & 3)) & 3; }
__host__ __device__ inline int RefTileW(int bx, int R) { return (2 * bx + 2 * R + RefTileShift(R) + 3) & ~3; }
__host__ __device__ inline int RefTileH(int bx, int tpp, int R) { return SweepRows(bx, tpp) + 2 * R; }
// Hypotheses per pixel of the sweep (K_NUM_SAMPS + 3, kernel_functions.h:32).
constexpr int kSweepHyp = 11;
// Largest dynamic shared memory a checkerboard block may request (the B200's
// 227 KB per block minus room for the kernels' static shared memory).
constexpr size_t kMaxDynamicSmem = 227 * 1024 - 2048;
// Dynamic shared memory of a sweep block: the reference tile (+128 bytes of
// alignment slack for the TMA destination), nb pose records, and per pixel the
// cost matrix, hypotheses, view weights and view probabilities.
__host__ __device__ inline size_t SweepKernelSmem(int R, int nb, int bx, int tpp) {
  const size_t P = tpp == 1 ? 0 : 256 / tpp;  // tpp == 1 keeps the per-pixel state in registers and local memory
  const size_t tile = (size_t)RefTileW(bx, R) * RefTileH(bx, tpp, R);
  return 128 + sizeof(float) * (tile + (size_t)nb * SMVS_POSE_FLOATS + P * (kSweepHyp * nb + kSweepHyp * 4 + 2 * nb));
}
// Same for a local-optimisation block (per pixel: five hypotheses' costs).
__host__ __device__ inline size_t LocalKernelSmem(int R, int nb, int bx, int tpp) {
  const size_t P = tpp == 1 ? 0 : 256 / tpp;
  const size_t tile = (size_t)RefTileW(bx, R) * RefTileH(bx, tpp, R);
  return 128 + sizeof(float) * (tile + (size_t)nb * SMVS_POSE_FLOATS + P * (5 * nb));
}
// Same for an InitConf block (32 x 8 pixels, one thread each: the cost vector
// and its sort order per pixel).
__host__ __device__ inline size_t InitConfKernelSmem(int R, int nb) {
  return sizeof(float) * ((size_t)(32 + 2 * R) * (8 + 2 * R) + (size_t)nb * SMVS_POSE_FLOATS + 2 * (size_t)nb * 256);
}
// Whether (bx, tpp) is a valid checkerboard launch shape.
inline bool ValidSweepShape(int bx, int tpp) {
  return (bx == 8 || bx == 16 || bx == 32 || bx == 64) && (tpp == 1 || tpp == 2 || tpp == 4) && bx * tpp <= 256;
}

// Encodes the TMA descriptor of a dense W x H FP32 reference image for the
// checkerboard tile of launch shape bx and window R. Returns false (use plain
// loads) when the image rows are not a multiple of 16 bytes, the image is
// smaller than the box, or the driver does not provide the encoder.
bool EncodeRefMap(CUtensorMap* map, const float* ref, int W, int H, int bx, int tpp, int R);

// All launchers enqueue on `stream` and return the launch status.
cudaError_t LaunchConvertImage(const void* in, int in_format, size_t in_stride, int w, int h, void* out,
                               int out_storage, size_t out_pitch, int normalise, cudaStream_t stream);
cudaError_t LaunchPrepRef(const JobParams& p, float* ref_sum, float* ref_sqsum, float* grad, cudaStream_t stream);
cudaError_t LaunchInit(const JobParams& p, int random_init, float opt_dmin, float opt_dmax, cudaStream_t stream);
// Propagate-depth initial maps (InitWorkspace, patch_match_cuda.cu:603-659):
// projects the depth map of every source with a map (src_depth[i], pitched
// device memory of row pitch src_pitch[i]; NULL = none) into `composite`
// (N*W*H floats of scratch), writes the median depths into p.depth where it is
// <= 0 and the consistent medians into `prior` (W*H, cleared first), then fits
// p.normal to p.depth. src_w/src_h: the sources' sizes (the projection grid is
// the largest of them).
cudaError_t LaunchPropagateInit(const JobParams& p, const int* src_w, const int* src_h, const float* const* src_depth,
                                const size_t* src_pitch, float* composite, float* prior, cudaStream_t stream);
// Batched checkerboard kernels: every job of `b` in one launch.
cudaError_t LaunchInitConf(const Batch& b, cudaStream_t stream);
cudaError_t LaunchSweep(const Batch& b, int colour, cudaStream_t stream);
cudaError_t LaunchLocalOpt(const Batch& b, int colour, cudaStream_t stream);
// iters[j] += 1 for every job of the batch (after both colours of an iteration).
cudaError_t LaunchAdvance(int* iters, int num_jobs, cudaStream_t stream);
// Views per pixel the checkerboard kernels reserve in shared memory for N
// source views (N rounded up to a multiple of 4); batches group jobs by it.
int ViewBucket(int N);
// The smallest tpp >= `tpp` whose sweep block fits in shared memory for nb
// views (results do not depend on it); 0 if none does.
int FitThreadsPerPixel(int R, int nb, int bx, int tpp);
// Test hook: at most this many blocks in persistent launches built from now on
// (0 = the resident count).
int PersistentGridCap();
void SetPersistentGridCap(int max_blocks);
// Opt every checkerboard kernel into large dynamic shared memory on the
// current device. Called once per device by the engine and the pool before
// any launch (and before any stream capture).
cudaError_t ConfigureKernels();
cudaError_t LaunchMask(const JobParams& p, const uint8_t* mask, cudaStream_t stream);
cudaError_t LaunchCurvature(const JobParams& p, uint16_t* curv, cudaStream_t stream);
cudaError_t LaunchGeomGradient(const JobParams& p, float* ggrad, cudaStream_t stream);
cudaError_t LaunchMedianFilter(const JobParams& p, const float* ggrad, float diff_thres, int colour, cudaStream_t stream);
cudaError_t LaunchConfFilter(const JobParams& p, float depth_thres, float conf_thres, int colour, cudaStream_t stream);
cudaError_t LaunchFilterDepthMaps(const JobParams& p, const float* in_depth, float* out_depth, int min_consistent,
                                  float filter_max_cost, int dedup, cudaStream_t stream);

bool SupportedWindow(int R, int S);

}  // namespace smvs
