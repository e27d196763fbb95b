// smvs_sweep.cuh — window-templated PatchMatch kernels (internal).
//
// Checkerboard kernels with G threads per pixel (G = 1, 2 or 4, a launch-shape
// knob). Per block (256 threads, 256 / G pixels): the reference-image tile the
// window needs and the N pose records are staged in shared memory once;
// source views are fetched through per-view texture objects over pitched HBM
// (hardware bilinear, border = 0, the sampling the reference configures at
// patch_match_cuda.cu:258-278). A pixel's cost matrix (hypotheses x views),
// its hypothesis list and its view weights live in shared memory, not in
// per-thread local memory. The G lanes of a pixel split the window rows of
// every NCC evaluation and add their partial moments with warp shuffles; all
// other per-pixel work is done identically by the G lanes (same inputs, same
// RNG draws), and lane 0 writes shared and global memory. The moments are
// always summed in one canonical order (rows by index mod 4 into four partial
// sums, combined as (p0 + p1) + (p2 + p3)), whatever G is, so maps do not
// depend on the launch shape. RNG draws come from a counter-based generator,
// so there is no per-pixel state array. Each supported (radius, step) pair is
// instantiated in its own translation unit (smvs_win_<R>_<S>.cu).
#pragma once

#include "smvs_device.cuh"
#include "smvs_kernels.h"

namespace smvs {
namespace detail {
namespace {  // internal linkage: every window translation unit gets its own copy

constexpr int kThreads = 256;  // threads per checkerboard block

__constant__ float kMWeights[5] = {0.f, 1.f, 2.01f, 3.03f, 4.06f};  // kernel_functions.cu:22
__constant__ int kNeighborOffs[4][2] = {{0, -1}, {-1, 0}, {0, 1}, {1, 0}};  // :23-25 (first four)
__constant__ int kDirSamples[8][20] = {  // :27-44 (row offset, col offset) pairs
    {-1, -2, 1, -2, -2, -3, 2, -3, -3, -4, 3, -4, -4, -5, 4, -5, -5, -6, 5, -6},
    {-1, 2, 1, 2, -2, 3, 2, 3, -3, 4, 3, 4, -4, 5, 4, 5, -5, 6, 5, 6},
    {-2, -1, -2, 1, -3, -2, -3, 2, -4, -3, -4, 3, -5, -4, -5, 4, -6, -5, -6, 5},
    {2, -1, 2, 1, 3, -2, 3, 2, 4, -3, 4, 3, 5, -4, 5, 4, 6, -5, 6, 5},
    {0, -3, 0, -5, 0, -7, 0, -9, 0, -11, 0, -13, 0, -15, 0, -17, 0, -19, 0, -21},
    {0, 3, 0, 5, 0, 7, 0, 9, 0, 11, 0, 13, 0, 15, 0, 17, 0, 19, 0, 21},
    {-3, 0, -5, 0, -7, 0, -9, 0, -11, 0, -13, 0, -15, 0, -17, 0, -19, 0, -21, 0},
    {3, 0, 5, 0, 7, 0, 9, 0, 11, 0, 13, 0, 15, 0, 17, 0, 19, 0, 21, 0}};

__device__ __forceinline__ float RefAt(const float* ref, int W, int H, int r, int c) {
  return (r >= 0 && r < H && c >= 0 && c < W) ? __ldg(ref + (size_t)r * W + c) : 0.0f;
}

// Stage the reference tile rows [row0, row0+th) x cols [col0, col0+tw) (border 0)
// and the pose records in shared memory.
__device__ __forceinline__ void StageShared(const JobParams& p, float* tile, int row0, int col0, int th, int tw,
                                            float* poses) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;
  for (int i = tid; i < th * tw; i += nthr) {
    const int r = i / tw, c = i - (i / tw) * tw;
    tile[i] = RefAt(p.ref, p.W, p.H, row0 + r, col0 + c);
  }
  for (int i = tid; i < p.N * SMVS_POSE_FLOATS; i += nthr) poses[i] = __ldg(p.poses + i);
}

// Bounded waits (mbarrier polls) before a kernel gives up on a TMA copy.
constexpr uint32_t kTmaWaitPolls = 1u << 22;

__device__ __forceinline__ float* Align128(float* p) {
  return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(p) + 127) & ~static_cast<uintptr_t>(127));
}

__device__ __forceinline__ uint32_t SmemAddr(const void* ptr) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(ptr));
}

__device__ __forceinline__ bool MbarPoll(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ bool MbarWait(uint32_t bar, uint32_t parity, uint32_t polls) {
  for (uint32_t i = 0; i < polls; ++i) {
    if (MbarPoll(bar, parity)) return true;
    if (i >= 32) __nanosleep(64);
  }
  return false;
}

// The block's reference tile as one TMA load: box (RefTileW x RefTileH) of
// `map` at column x (a multiple of 4) and row y into `tile` (128-byte aligned
// shared memory); rows and columns outside the image read as zero (the
// border of the reference's texture). `uses` counts the block's earlier
// loads (block-uniform): the first one initialises the mbarrier, and load k
// completes the barrier's phase k, so a persistent block reuses one barrier
// for all its tiles. Every thread waits with a bounded wait (`polls`). Returns
// false after setting *status if the copy did not land; the caller then leaves
// the block's pixels unchanged and the block stops.
__device__ __forceinline__ bool TmaStageTile(const CUtensorMap* map, float* tile, int x, int y, uint32_t bytes,
                                             uint64_t* mbar, uint32_t& uses, int* status, uint32_t polls,
                                             bool skip_copy) {
  const uint32_t bar = SmemAddr(mbar);
  const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
  if (uses == 0) {
    if (leader) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  if (leader) {
    // The block's reads of the previous tile (ordered before this point by the
    // barrier that ended it) come before the copy that overwrites it.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    if (!skip_copy)
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
          ::"r"(SmemAddr(tile)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
          : "memory");
  }
  const uint32_t parity = uses & 1u;
  ++uses;
  const bool landed = MbarWait(bar, parity, polls);
  if (!__syncthreads_or(!landed)) return true;  // block-uniform outcome
  if (leader) atomicExch(status, 1);
  // Let a late copy land before the block's shared memory is released (no
  // copy is in flight when the test hook skipped it).
  if (!skip_copy) MbarWait(bar, parity, kTmaWaitPolls);
  return false;
}

// Stage the reference tile (TMA when the job has a descriptor for this launch
// shape, else plain loads) and the pose records. `tile` holds RefTileH rows of
// RefTileW floats starting at (row0 - R, col0 - R - RefTileShift(R)).
template <int R>
__device__ __forceinline__ bool StageRefTile(const Batch& b, int job, const JobParams& p, float* tile, int row0,
                                             int col0, int rows, float* poses, uint64_t* mbar, uint32_t& tma_uses) {
  const int bx = b.block_x;
  const int tw = RefTileW(bx, R), th = rows + 2 * R;
  const int x0 = col0 - R - RefTileShift(R), y0 = row0 - R;
  const bool tma = b.ref_maps != nullptr && p.tma_box_w == tw && p.tma_box_h == th;
  if (!tma) {
    StageShared(p, tile, y0, x0, th, tw, poses);
    return true;
  }
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = tid; i < p.N * SMVS_POSE_FLOATS; i += blockDim.x * blockDim.y) poses[i] = __ldg(p.poses + i);
  return TmaStageTile(b.ref_maps + job, tile, x0, y0, (uint32_t)(tw * th * sizeof(float)), mbar, tma_uses, b.status,
                      b.tma_polls > 0 ? (uint32_t)b.tma_polls : kTmaWaitPolls, b.tma_skip_copy != 0);
}

// Batched launches: find the job of tile `bid` (binary search over the tile
// prefix sums), read its iteration counter and stage its parameters in
// shared memory. Every thread of the block returns the same values.
__device__ __forceinline__ void DecodeBlock(const Batch& b, const int* prefix, int bid, JobParams& sp, int& job,
                                            int& blk, int& iter) {
  __shared__ int s_job, s_blk, s_iter;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    int lo = 0, hi = b.num_jobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(prefix + mid) <= bid) lo = mid; else hi = mid - 1;
    }
    s_job = lo;
    s_blk = bid - __ldg(prefix + lo);
    s_iter = b.iters ? b.iters[lo] : 0;
  }
  __syncthreads();
  job = s_job;
  blk = s_blk;
  iter = s_iter;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;
  const int4* src = reinterpret_cast<const int4*>(b.jobs + job);
  int4* dst = reinterpret_cast<int4*>(&sp);
  for (int i = tid; i < (int)(sizeof(JobParams) / sizeof(int4)); i += nthr) dst[i] = src[i];
  __syncthreads();
}

// The lanes of this thread's pixel: G consecutive lanes of the warp.
template <int G>
__device__ __forceinline__ unsigned GroupMask() {
  const unsigned lane = threadIdx.x & 31u;
  return (G == 1) ? (1u << lane) : (((1u << G) - 1u) << (lane & ~(unsigned)(G - 1)));
}

// Sum of the four row-class partials a[k] (k = the lane's k-th class) over the
// pixel's lanes, always as (p0 + p1) + (p2 + p3), where p_c is the sum over the
// window rows i with i mod 4 == c. Lane l of G owns classes l, l + G, ...
template <int G>
__device__ __forceinline__ float CombineClasses(const float* a, unsigned gmask) {
  if (G == 1) return (a[0] + a[1]) + (a[2] + a[3]);
  if (G == 2) {
    const float s01 = a[0] + __shfl_xor_sync(gmask, a[0], 1);
    const float s23 = a[1] + __shfl_xor_sync(gmask, a[1], 1);
    return s01 + s23;
  }
  const float s = a[0] + __shfl_xor_sync(gmask, a[0], 1);
  return s + __shfl_xor_sync(gmask, s, 2);
}

// ComputeNCCCost<R,S>, kernel_functions.cu:1245-1340, with the window rows
// split over the G lanes of the pixel (lane `lane` takes rows lane, lane + G,
// ...). `win` points at the window's top-left in the shared tile (row stride
// ws). The source positions follow the reference's incremental scheme exactly
// (row starts advanced by one row step at a time, taps by one column step);
// every lane returns the same value.
// kUnrollRows: unroll the row groups too when the window has at most 8 rows
// (step 2 or radius 3); measured on the 1600x1200, 10-view workload at step 2
// it shortens the init-conf and local-optimisation launches by 11 % and 8 % and
// lengthens the sweep's by 1 %, so those two kernels ask for it. The
// arithmetic and its order do not change.
template <int R, int S, int G, bool kUnrollRows = false>
__device__ __forceinline__ float NccCost(cudaTextureObject_t tex, const float* pose, int row, int col, float depth,
                                         const float n[3], const float iK[4], int W, int H, float center,
                                         float rsum, float rvar, const float* win, int ws, float sn, float cn,
                                         int lane, unsigned gmask) {
  constexpr float kMaxCost = 2.0f;
  constexpr int kRows = 2 * R / S + 1;
  constexpr int kClasses = 4 / G;  // row classes (mod 4) per lane
  float Hm[9];
  ComposeHomography(pose, row, col, depth, n, iK, Hm);
  const float inv_z0 = 1.0f / (Hm[6] * col + Hm[7] * row + Hm[8]);
  const int u = (int)((Hm[0] * col + Hm[1] * row + Hm[2]) * inv_z0);
  const int v = (int)((Hm[3] * col + Hm[4] * row + Hm[5]) * inv_z0);
  // [quirk] bounds are the reference image's width/height (:1265-1270).
  if (u < 0 || u >= W || v < 0 || v >= H) return kMaxCost;
  const int row_start = row - R, col_start = col - R;
  float bcol = Hm[0] * col_start + Hm[1] * row_start + Hm[2];
  float brow = Hm[3] * col_start + Hm[4] * row_start + Hm[5];
  float bz = Hm[6] * col_start + Hm[7] * row_start + Hm[8];
  const float h0 = S * Hm[0], h1 = S * Hm[1], h3 = S * Hm[3], h4 = S * Hm[4], h6 = S * Hm[6], h7 = S * Hm[7];
  for (int k = 0; k < lane; ++k) { bcol += h1; brow += h4; bz += h7; }  // this lane's first row
  float ss[kClasses], sss[kClasses], srs[kClasses], sw[kClasses];
#pragma unroll
  for (int k = 0; k < kClasses; ++k) { ss[k] = 0.f; sss[k] = 0.f; srs[k] = 0.f; sw[k] = 0.f; }
  // Rows in groups of four; within a group this lane takes rows q + lane + k G.
  // Taps of a row are unrolled; the groups stay rolled (instruction cache)
  // unless kUnrollRows asks otherwise for a short window.
  constexpr int kGroupUnroll = (kUnrollRows && kRows <= 8) ? (kRows + 3) / 4 : 1;
#pragma unroll kGroupUnroll
  for (int q = 0; q < kRows; q += 4) {
#pragma unroll
    for (int k = 0; k < kClasses; ++k) {
      const int i = q + lane + k * G;
      if (i < kRows) {
        const int dr = -R + i * S;
        const float* wrow = win + (dr + R) * ws + R;
        const float sr = (float)(dr * dr);
        float col_src = bcol, row_src = brow, z = bz;
#pragma unroll
        for (int dc = -R; dc <= R; dc += S) {
          const float iz = 1.0f / z;
          const float fu = iz * col_src + 0.5f;
          const float fv = iz * row_src + 0.5f;
          const float rc = wrow[dc];
          const float sc = tex2D<float>(tex, fu, fv);
          const float cd = center - rc;
          const float wgt = __expf(-(sr + (float)(dc * dc)) * sn - cd * cd * cn);
          const float wsc = wgt * sc;
          ss[k] += wsc;
          sss[k] += wsc * sc;
          srs[k] += wsc * rc;
          sw[k] += wgt;
          col_src += h0;
          row_src += h3;
          z += h6;
        }
      }
#pragma unroll
      for (int t = 0; t < G; ++t) { bcol += h1; brow += h4; bz += h7; }
    }
  }
  float tss = CombineClasses<G>(ss, gmask);
  float tsss = CombineClasses<G>(sss, gmask);
  float tsrs = CombineClasses<G>(srs, gmask);
  const float tsw = CombineClasses<G>(sw, gmask);
  const float isw = 1.0f / tsw;
  tss *= isw; tsss *= isw; tsrs *= isw;
  const float svar = tsss - tss * tss;
  if (rvar < 1e-5f || svar < 1e-5f) return kMaxCost;
  const float cov = tsrs - rsum * tss;
  const float val = 1.0f - cov * rsqrtf(rvar * svar);
  return fmaxf(0.0f, fminf(kMaxCost, val));
}

struct PixRef {
  float center, rsum, rvar;
  const float* win;
  int ws;
};

// A pixel's prior (SweepOptions::prior_depth_ncc / propagate_depth): depth w,
// normal xyz and weight, read where the reference reads them
// (kernel_functions.cu:1533-1543, 2188-2200); a NULL map reads as 0.
struct PriorInfo {
  float x, y, z, w, wgt;
};

__device__ __forceinline__ PriorInfo LoadPrior(const JobParams& p, size_t pix) {
  PriorInfo pi = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (p.prior_mode == 0) return pi;
  const size_t WH = (size_t)p.W * p.H;
  pi.w = p.prior_depth[pix];
  if (p.prior_normal) {
    pi.x = p.prior_normal[pix];
    pi.y = p.prior_normal[WH + pix];
    pi.z = p.prior_normal[2 * WH + pix];
  }
  if (p.prior_wgt) pi.wgt = p.prior_wgt[pix];
  return pi;
}

// The factor ComputeMultiViewCostVector applies to every NCC cost of a
// hypothesis (kernel_functions.cu:1470-1478): ComputeNCCWeightFromPrior
// (:316-340), which lowers the cost of hypotheses near the prior depth and
// normal, times 1 - 0.3 wgt for a weight strictly between 0 and 1. It is 1
// unless the job has a prior depth and normal (mode 1) and the pixel's prior
// depth is above FLT_EPSILON. The reference's mixed float/double arithmetic is
// kept: the colour-variance term and the factors are double, the exponentials
// of the depth and angle terms single precision.
__device__ __forceinline__ float PriorWeight(const JobParams& p, const PriorInfo& pi, const float h[3], float hd,
                                             float rvar) {
  if (p.prior_mode != 1 || !(pi.w > FLT_EPSILON)) return 1.0f;
  float regu = 1.0f;
  const float sigma2 = (float)(0.5 - 0.4 * exp(-10000.0 * (double)fabsf(rvar)));
  const float dd = hd - pi.w;
  const float dd2 = fmaxf(dd * dd, 0.05f * 0.05f);
  regu = (float)((double)regu * fmax(1.0 - 0.2 * (double)__expf(-dd2 / sigma2), 0.01));
  const float pn = pi.x * pi.x + pi.y * pi.y + pi.z * pi.z;
  if ((double)pn > 0.8 && (double)pn < 1.25) {
    const float ct = pi.x * h[0] + pi.y * h[1] + pi.z * h[2];
    const float dt2 = (1.0f - ct) * (1.0f - ct);
    regu = (float)((double)regu * fmax(1.0 - 0.54 * (double)__expf(-dt2 / sigma2), 0.01));
  }
  if ((double)pi.wgt < 1.0 && (double)pi.wgt > 0.0) regu = (float)((double)regu * (1.0 - (double)pi.wgt * 0.3));
  return regu;
}

// Cost of one hypothesis on source view v: the NCC cost times the prior
// factor pw (1 without a prior), plus the weighted geometric term.
template <int R, int S, int G, bool kUnrollRows = false>
__device__ __forceinline__ float ViewCost(const JobParams& p, const float* poses, int v, int row, int col,
                                          float depth, const float n[3], const float np[3], const PixRef& pr,
                                          const float* Kgeom, int lane, unsigned gmask, float pw = 1.0f) {
  const float* pose = poses + v * SMVS_POSE_FLOATS;
  float cost = NccCost<R, S, G, kUnrollRows>(p.src_tex[v], pose, row, col, depth, n, p.refiK, p.W, p.H, pr.center, pr.rsum,
                                pr.rvar, pr.win, pr.ws, p.sn, p.cn, lane, gmask);
  if (pw != 1.0f) cost *= pw;  // keeps the no-prior arithmetic (and any contraction) unchanged
  if (p.geom)
    cost += p.geom_reg * GeomCost(pose, p.dep_tex[v], (float)row, (float)col, depth, np, Kgeom, p.geom_max);
  return cost;
}

// InitConfMapKernel, kernel_functions.cu:1497-1601. One thread per
// pixel; the cost vector and its sort order live in shared memory
// ([view][pixel], nb views per pixel).
template <int R, int S>
__global__ void __launch_bounds__(kThreads) InitConfKernel(const Batch b) {
  extern __shared__ float smem[];
  __shared__ JobParams sp;
  int job, blk, iter;
  DecodeBlock(b, b.conf_block_start, blockIdx.x, sp, job, blk, iter);
  const JobParams& p = sp;
  const int kBX = blockDim.x, kBY = blockDim.y;
  const int tw = kBX + 2 * R, th = kBY + 2 * R;
  const int nb = b.NB;
  float* tile = smem;
  float* poses = smem + tw * th;
  float* costs = poses + nb * SMVS_POSE_FLOATS;
  int* order = reinterpret_cast<int*>(costs + nb * kThreads);
  const int col0 = (blk % p.conf_blocks_x) * kBX, row0 = (blk / p.conf_blocks_x) * kBY;
  StageShared(p, tile, row0 - R, col0 - R, th, tw, poses);
  __syncthreads();
  const int col = col0 + threadIdx.x, row = row0 + threadIdx.y;
  if (col >= p.W || row >= p.H) return;
  const int t = threadIdx.y * kBX + threadIdx.x;
  const size_t WH = (size_t)p.W * p.H;
  const size_t pix = (size_t)row * p.W + col;
  PixRef pr;
  pr.center = p.ref[pix];
  pr.rsum = p.ref_sum[pix];
  pr.rvar = p.ref_sqsum[pix] - pr.rsum * pr.rsum;
  pr.ws = tw;
  pr.win = tile + threadIdx.y * tw + threadIdx.x;
  const float np[3] = {p.refiK[0] * col + p.refiK[1], p.refiK[2] * row + p.refiK[3], 1.0f};
  const float n[3] = {p.normal[pix], p.normal[WH + pix], p.normal[2 * WH + pix]};
  const float depth = p.depth[pix];
  const unsigned gmask = GroupMask<1>();
  const float pw = PriorWeight(p, LoadPrior(p, pix), n, depth, pr.rvar);
#define C_(v) costs[(v) * kThreads + t]
#define O_(v) order[(v) * kThreads + t]
  for (int v = 0; v < p.N; ++v) {
    const float c = ViewCost<R, S, 1, true>(p, poses, v, row, col, depth, n, np, pr, p.refK, 0, gmask, pw);
    C_(v) = c;
    O_(v) = v;
    p.cost[(size_t)v * WH + pix] = c;
  }
  // Partial bubble sort: only the best thk positions are needed and the
  // reference's full ascending bubble sort (utils.h:212-231) puts the same
  // (stable) values there.
  for (int i = 0; i < p.N - 1; ++i)
    for (int j = 0; j < p.N - 1 - i; ++j)
      if (C_(j) > C_(j + 1)) {
        const float tc = C_(j); C_(j) = C_(j + 1); C_(j + 1) = tc;
        const int to = O_(j); O_(j) = O_(j + 1); O_(j + 1) = to;
      }
  float conf = 0.f;
  uint32_t sel = p.view_sel[pix];
  for (int i = 0; i < p.thk; ++i) { conf += C_(i); sel |= (1u << O_(i)); }
#undef C_
#undef O_
  conf /= kMWeights[p.thk];
  p.conf[pix] = conf;
  p.view_sel[pix] = sel;
}

// Shared-memory layout of a checkerboard block after the reference tile and
// the pose records (floats, P pixels, nb views per pixel, pixel index fastest).
struct SweepSmem {
  float* M;   // [kMaxHyp][nb][P]  cost of hypothesis h on view v
  float* HY;  // [kMaxHyp][4][P]   hypotheses (normal xyz, depth)
  float* VW;  // [nb][P]           view weights
  float* PR;  // [nb][P]           view probabilities, then their CDF
};

// Threads-per-pixel 1: the thread-per-pixel form of SweepFromCheckerBoardOpt
// (kernel_functions.cu:2136-2560, with the prior and propagate-depth paths)
// and LocalOptimization (:2736-2931). The
// pixel's cost matrix M[kMaxHyp][NB], its hypotheses and view weights are
// per-thread arrays (NB = the view bucket): the compiler keeps them in the
// thread's local frame, which lives in the L1 next to the texture cache the
// cost windows read. Measured on the 1600x1200, 10-view workload this is the
// fastest layout: keeping those arrays in shared memory shrinks the L1 that the
// texture fetches need (the G = 2 / 4 kernels below), and keeping them in an
// L2-resident global scratch makes the scalar phases wait on L2 latency. The
// arithmetic is the same as the G-lane kernels (NccCost<R,S,1> sums the window
// in the same canonical order), so maps are identical for every
// threads-per-pixel value.
// Resident blocks per SM the thread-per-pixel kernels ask the register
// allocator for: at window step 2 with up to 16 views the launch is
// latency-bound and a third block (80 registers, a few spills) is measured
// 2-3 % faster (10 views); otherwise the allocator's own choice (128 registers,
// two blocks) is kept (0 = no bound).
template <int S, int NB>
struct ThreadPixelBlocks {
  static constexpr int kMin = (S == 2 && NB <= 16) ? 3 : 0;
};

template <int R, int S, int NB>
__device__ __forceinline__ bool SweepTileL(const Batch& b, int colour, int bid, float* smem, JobParams& sp,
                                           uint64_t* mbar, uint32_t& tma_uses) {
  int job, blk, iter;
  DecodeBlock(b, b.block_start, bid, sp, job, blk, iter);
  const JobParams& p = sp;
  if (iter >= p.num_iterations) return true;  // finished job of the batch (block-uniform)
  const float th_mc = p.th_tab[iter];
  const uint64_t skey = StageKey(p.seed, StageSweep(iter, colour));
  const int kBX = b.block_x, kBY = kThreads / b.block_x;
  const int tw = RefTileW(kBX, R), th = kBY + 2 * R;
  float* tile = Align128(smem);  // a TMA destination starts on a 128-byte boundary
  float* poses = tile + tw * th;
  const int col0 = (blk % p.blocks_x) * 2 * kBX, row0 = (blk / p.blocks_x) * kBY;
  if (!StageRefTile<R>(b, job, p, tile, row0, col0, kBY, poses, mbar, tma_uses)) return false;  // block-uniform
  __syncthreads();
  const int tx = threadIdx.x % kBX, ty = threadIdx.x / kBX;
  const int row = row0 + ty;
  const int col = col0 + 2 * tx + ((row + colour) & 1);
  if (col >= p.W || row >= p.H) return true;
  const int W = p.W, H = p.H, N = p.N;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  const unsigned gmask = GroupMask<1>();
  Rng r(skey, (uint32_t)pix);
  float depth = p.depth[pix];
  float normal[3] = {p.normal[pix], p.normal[WH + pix], p.normal[2 * WH + pix]};
  const float grad = p.grad[pix];
  const PriorInfo pri = LoadPrior(p, pix);
  // A prior depth narrows the random normal perturbation (:2201-2203, 2213-2214).
  const float prf = (p.prior_mode == 1 && (double)pri.w > 1e-6) ? 0.1f : 1.0f;
  const float depth_min = p.depth_min;
  const float depth_max = (float)(1.2 * (double)p.depth_max);  // [quirk] :2213
  const float a1 = fminf(p.rand_a1 * prf, (float)(180.0 * 0.0174532925199432));
  const float a2 = fminf(p.rand_a2 * prf, (float)(90.0 * 0.0174532925199432));
  const float* iK = p.refiK;
  const float vd[3] = {iK[0] * col + iK[1], iK[2] * row + iK[3], 1.0f};
  const float ivl = rsqrtf(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);

  float hyp[kMaxHyp][4];
  int ns = 0;
  hyp[0][0] = normal[0]; hyp[0][1] = normal[1]; hyp[0][2] = normal[2]; hyp[0][3] = depth;
  ns = 1;
  if (grad >= 1.0f) {  // :2237-2276
    float nconf[4], O[4];
    int nvalid = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      O[i] = (float)i;
      const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
      if (u < 0 || u >= W || v < 0 || v >= H) { nconf[i] = FLT_MAX; continue; }
      nvalid++;
      nconf[i] = p.conf[(size_t)v * W + u];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3 - i; ++j)
        if (nconf[j] > nconf[j + 1]) {
          float t = nconf[j]; nconf[j] = nconf[j + 1]; nconf[j + 1] = t;
          t = O[j]; O[j] = O[j + 1]; O[j + 1] = t;
        }
    nvalid = min(nvalid, 2);
    for (int i = 0; i < nvalid; ++i) {
      const int idx = (int)O[i];
      const int u = kNeighborOffs[idx][1] + col, v = kNeighborOffs[idx][0] + row;
      const size_t q = (size_t)v * W + u;
      float nn[3] = {p.normal[q], p.normal[WH + q], p.normal[2 * WH + q]};
      CorrectNormal(nn, vd, ivl);
      hyp[ns][3] = PropagateDepth(p.depth[q], nn, iK, v, u, vd);
      hyp[ns][0] = nn[0]; hyp[ns][1] = nn[1]; hyp[ns][2] = nn[2];
      ns++;
    }
  }
  for (int k = 0; k < 8; ++k) {  // :2278-2327
    int br = 0, bc = 0;
    float best = FLT_MAX;
#pragma unroll
    for (int s = 0; s < 10; ++s) {
      const int nr = row + kDirSamples[k][2 * s], nc = col + kDirSamples[k][2 * s + 1];
      if (nr < 0 || nr >= H || nc < 0 || nc >= W) continue;
      float nconf = p.conf[(size_t)nr * W + nc];
      if (p.prior_mode != 0 && p.prior_wgt) {  // PRIOR_WGT_PROGET, :2292-2304
        const float pws = p.prior_wgt[(size_t)nr * W + nc];
        if ((double)pws > 1e-6) nconf = (float)((double)nconf * (1.0 - 0.2 * (double)pws));
      }
      if (best > nconf) { br = nr; bc = nc; best = nconf; }
    }
    if (best < FLT_MAX) {
      const size_t q = (size_t)br * W + bc;
      float nn[3] = {p.normal[q], p.normal[WH + q], p.normal[2 * WH + q]};
      CorrectNormal(nn, vd, ivl);
      hyp[ns][3] = PropagateDepth(p.depth[q], nn, iK, br, bc, vd);
      hyp[ns][0] = nn[0]; hyp[ns][1] = nn[1]; hyp[ns][2] = nn[2];
      ns++;
    }
  }

  PixRef pr;
  pr.center = p.ref[pix];
  pr.rsum = p.ref_sum[pix];
  pr.rvar = p.ref_sqsum[pix] - pr.rsum * pr.rsum;
  pr.ws = tw;
  pr.win = tile + ty * tw + (col - col0) + RefTileShift(R);
  float M[kMaxHyp][NB];
  for (int v = 0; v < N; ++v) M[0][v] = p.cost[(size_t)v * WH + pix];
  float vw[NB];
  float costs[kMaxHyp];
  // Two evaluation phases share one call site of the cost code: phase 0 scores
  // the propagated hypotheses 1..ns-1, phase 1 the refinement hypotheses 1..4.
  int h_end = ns;
  for (int phase = 0; phase < 2; ++phase) {
    for (int h = 1; h < h_end; ++h) {
      const float pw = PriorWeight(p, pri, hyp[h], hyp[h][3], pr.rvar);
      for (int v = 0; v < N; ++v)
        M[h][v] = ViewCost<R, S, 1>(p, poses, v, row, col, hyp[h][3], hyp[h], vd, pr, p.refK, 0, gmask, pw);
    }
    if (phase == 1) break;

    // ACMM view selection, :2364-2427.
    uint32_t flags = 0;
    float probs[NB];
    for (int v = 0; v < N; ++v) {
      unsigned n1 = 0, n2 = 0;
      float pv = 0.f;
      for (int h = 0; h < ns; ++h) {
        const float cst = M[h][v];
        pv += __expf(-cst * cst * p.inv_beta2);
        n1 += (cst < th_mc);
        n2 += (cst > p.max_mc);
      }
      probs[v] = pv;
      if ((int)n1 >= p.num_good && (int)n2 <= p.num_bad) flags |= (1u << v);
    }
    if (flags == 0) return true;
    for (int v = 0; v < N; ++v)
      if (!((flags >> v) & 1u)) probs[v] = 0.f;
    {
      float sum = 0.f;
      for (int v = 0; v < N; ++v) sum += probs[v];
      const float inv = 1.0f / sum;
      float cum = 0.f;
      for (int v = 0; v < N; ++v) { cum += probs[v] * inv; probs[v] = cum; }
    }
    for (int v = 0; v < N; ++v) vw[v] = 0.f;
    for (int s = 0; s < p.num_samples; ++s) {
      const float rp = r.Uniform() - FLT_EPSILON;
      for (int v = 0; v < N; ++v)
        if (probs[v] > rp) {
          if (p.random_opt) vw[v] = 1.0f; else vw[v] += 1.0f;
          break;
        }
    }
    float wn = 0.f;
    for (int v = 0; v < N; ++v) wn += vw[v];
    if (wn <= 1e-5f) return true;
    const float iwn = 1.0f / wn;
    uint32_t sel = 0;
    for (int v = 0; v < N; ++v) { vw[v] *= iwn; if (vw[v] > 0) sel |= (1u << v); }
    for (int h = 0; h < ns; ++h) {
      float cs = 0.f;
      for (int v = 0; v < N; ++v) cs += vw[v] * M[h][v];
      costs[h] = cs;
    }
    p.view_sel[pix] = sel;
    int mi = -1;
    if (p.prior_mode == 1 && pri.w > 0.0f) {
      // FindMinCostWithin (:661-671) over the band the prior allows
      // (:2431-2437; [quirk] the lower end is min(0.95 w - 0.05, 0)).
      const float lo = (float)fmin((double)(pri.w * 0.95f) - 0.05, 0.0);
      const float hi = (float)((double)(pri.w * 1.05f) + 0.05);
      float m = FLT_MAX;
      for (int h = 0; h < ns; ++h)
        if (costs[h] <= m && hyp[h][3] >= lo && hyp[h][3] <= hi) { m = costs[h]; mi = h; }
    } else {
      float m = FLT_MAX;
      for (int h = 0; h < ns; ++h)
        if (costs[h] <= m) { m = costs[h]; mi = h; }  // FindMinCost :648-659 ('<=')
    }
    if (mi < 0) return true;
    depth = hyp[mi][3];
    normal[0] = hyp[mi][0]; normal[1] = hyp[mi][1]; normal[2] = hyp[mi][2];
    if (mi != 0)
      for (int v = 0; v < N; ++v) M[0][v] = M[mi][v];

    // Refinement hypotheses, :2449-2486.
    float nn[3];
    const float pd_min = (1.0f - p.rand_depth_ratio) * depth, pd_max = (1.0f + p.rand_depth_ratio) * depth;
    const float ndepth = r.Uniform() * (pd_max - pd_min) + pd_min;  // PerturbDepth :141-147
    PerturbNormalACMH(normal, nn, a1, a2, r);
    CorrectNormal(nn, vd, ivl);
    // With propagate_depth a pixel that has a prior depth gets no random
    // depth hypothesis (:2467-2486).
    const bool rand_depth = !(p.prior_mode == 2 && pri.w > 0.0f);
    const float rdepth = rand_depth ? r.Uniform() * (depth_max - depth_min) + depth_min : 0.0f;
    float rn[3];
    RandomNormal(r, vd, rn);
    CorrectNormal(rn, vd, ivl);
    hyp[0][0] = normal[0]; hyp[0][1] = normal[1]; hyp[0][2] = normal[2]; hyp[0][3] = depth;
    hyp[1][0] = nn[0]; hyp[1][1] = nn[1]; hyp[1][2] = nn[2]; hyp[1][3] = depth;
    hyp[2][0] = normal[0]; hyp[2][1] = normal[1]; hyp[2][2] = normal[2]; hyp[2][3] = ndepth;
    hyp[3][0] = rn[0]; hyp[3][1] = rn[1]; hyp[3][2] = rn[2]; hyp[3][3] = depth;
    hyp[4][0] = normal[0]; hyp[4][1] = normal[1]; hyp[4][2] = normal[2]; hyp[4][3] = rdepth;
    h_end = rand_depth ? 5 : 4;
  }
  // :2488-2559: weighted refinement costs, argmin, write back.
  for (int h = 0; h < h_end; ++h) {
    float cs = 0.f;
    for (int v = 0; v < N; ++v) cs += vw[v] * M[h][v];
    costs[h] = cs;
  }
  int mi = -1;
  {
    float m = FLT_MAX;
    for (int h = 0; h < h_end; ++h)
      if (costs[h] <= m) { m = costs[h]; mi = h; }
  }
  if (mi != -1) {
    p.conf[pix] = costs[mi];
    p.depth[pix] = hyp[mi][3];
    p.normal[pix] = hyp[mi][0]; p.normal[WH + pix] = hyp[mi][1]; p.normal[2 * WH + pix] = hyp[mi][2];
    for (int v = 0; v < N; ++v) p.cost[(size_t)v * WH + pix] = M[mi][v];
  }
  return true;
}

// One block per checkerboard tile, or a persistent grid (resident blocks per
// SM x SMs) whose blocks stride over the tiles: a tile's pixels read only
// the other colour's state, so the tile order never changes results. The
// per-pixel arithmetic is the same code in both launch forms.
template <int R, int S, int NB>
__global__ void __launch_bounds__(kThreads, ThreadPixelBlocks<S, NB>::kMin) SweepKernelL(const Batch b, int colour) {
  extern __shared__ float smem[];
  __shared__ JobParams sp;
  __shared__ uint64_t mbar;
  uint32_t tma_uses = 0;
  for (int t = blockIdx.x; t < b.total_blocks; t += gridDim.x) {
    if (!SweepTileL<R, S, NB>(b, colour, t, smem, sp, &mbar, tma_uses)) return;
    __syncthreads();  // the tile's shared memory is free for the next tile
  }
}

// One block per checkerboard tile. (This kernel is kept out of the
// persistent form: restructured as a tile loop its code generation rounds a
// few normals differently in the last bit from LocalOptKernel<R, S, G>.)
template <int R, int S, int NB>
__global__ void __launch_bounds__(kThreads, ThreadPixelBlocks<S, NB>::kMin) LocalOptKernelL(const Batch b, int colour) {
  extern __shared__ float smem[];
  __shared__ JobParams sp;
  __shared__ uint64_t mbar;
  int job, blk, iter;
  DecodeBlock(b, b.block_start, blockIdx.x, sp, job, blk, iter);
  const JobParams& p = sp;
  // Iterations > 2 only (patch_match_cuda.cu:861-880); block-uniform.
  if (iter >= p.num_iterations || !p.local_opt || iter <= 2) return;
  const uint64_t skey = StageKey(p.seed, StageLocal(iter, colour));
  const int kBX = b.block_x, kBY = kThreads / b.block_x;
  const int tw = RefTileW(kBX, R), th = kBY + 2 * R;
  float* tile = Align128(smem);  // a TMA destination starts on a 128-byte boundary
  float* poses = tile + tw * th;
  const int col0 = (blk % p.blocks_x) * 2 * kBX, row0 = (blk / p.blocks_x) * kBY;
  uint32_t tma_uses = 0;
  if (!StageRefTile<R>(b, job, p, tile, row0, col0, kBY, poses, &mbar, tma_uses)) return;  // block-uniform
  __syncthreads();
  const int tx = threadIdx.x % kBX, ty = threadIdx.x / kBX;
  const int row = row0 + ty;
  const int col = col0 + 2 * tx + ((row + colour) & 1);
  if (col >= p.W || row >= p.H) return;
  const int W = p.W, H = p.H, N = p.N;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  const unsigned gmask = GroupMask<1>();
  Rng r(skey, (uint32_t)pix);
  float conf = p.conf[pix];
  float depth = p.depth[pix];
  float normal[3] = {p.normal[pix], p.normal[WH + pix], p.normal[2 * WH + pix]};
  const uint32_t sel = p.view_sel[pix];
  const float a1 = (float)(4.0 * 0.0174532925199432), a2 = (float)(2.0 * 0.0174532925199432);
  const float* iK = p.refiK;
  const float np[3] = {iK[0] * col + iK[1], iK[2] * row + iK[3], 1.0f};
  float m[3] = {normal[0], normal[1], normal[2]};
  float lo = depth, hi = depth;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
    if (u < 0 || u >= W || v < 0 || v >= H) continue;
    const size_t q = (size_t)v * W + u;
    const float nd = p.depth[q];
    m[0] += p.normal[q]; m[1] += p.normal[WH + q]; m[2] += p.normal[2 * WH + q];
    if (nd <= lo) lo = nd;
    if (nd > hi) hi = nd;
  }
  const float inv_norm = rsqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  m[0] *= inv_norm; m[1] *= inv_norm; m[2] *= inv_norm;
  PixRef pr;
  pr.center = p.ref[pix];
  pr.rsum = p.ref_sum[pix];
  pr.rvar = p.ref_sqsum[pix] - pr.rsum * pr.rsum;
  pr.ws = tw;
  pr.win = tile + ty * tw + (col - col0) + RefTileShift(R);
  float M[5][NB];
  float hyp[5][4];
  int mi = -1;
  // Rounds 0..4 score five random hypotheses on the selected views; round 5
  // rescores the winner on the unselected views. One call site of the cost code.
  for (int it = 0; it < 6; ++it) {
    float hcur[4];
    if (it < 5) {
      hyp[it][3] = r.Uniform() * (hi - lo) + lo;
      PerturbNormalACMH(m, hyp[it], a1, a2, r);
      hcur[0] = hyp[it][0]; hcur[1] = hyp[it][1]; hcur[2] = hyp[it][2]; hcur[3] = hyp[it][3];
    } else {
      if (mi == -1) break;
      hcur[0] = normal[0]; hcur[1] = normal[1]; hcur[2] = normal[2]; hcur[3] = depth;
    }
    // [quirk] :2916-2919 passes the inverse intrinsics where K is expected when
    // rescoring the unselected views.
    const float* Kg = (it < 5) ? p.refK : p.refiK;
    float mconf = 0.f, mw = 0.f;
    for (int v = 0; v < N; ++v) {
      const bool selected = (sel >> v) & 1u;
      if (selected != (it < 5)) continue;
      const float cost = ViewCost<R, S, 1, true>(p, poses, v, row, col, hcur[3], hcur, np, pr, Kg, 0, gmask);
      if (it < 5) {
        M[it][v] = cost;
        mconf += cost;
        mw += 1.f;
      } else {
        p.cost[(size_t)v * WH + pix] = cost;
      }
    }
    if (it == 5) break;
    if (mw <= 0.f) return;
    mconf /= mw;
    if (mconf < conf) {
      conf = mconf;
      depth = hyp[it][3];
      normal[0] = hyp[it][0]; normal[1] = hyp[it][1]; normal[2] = hyp[it][2];
      mi = it;
    }
  }
  if (mi != -1) {
    p.conf[pix] = conf;
    p.depth[pix] = depth;
    p.normal[pix] = normal[0]; p.normal[WH + pix] = normal[1]; p.normal[2 * WH + pix] = normal[2];
    for (int v = 0; v < N; ++v)
      if ((sel >> v) & 1u) p.cost[(size_t)v * WH + pix] = M[mi][v];
  }
}

// Blocks per SM the register allocation must allow: shared memory holds one
// block per SM at G = 1 (10 views), two at G = 2 and three at G = 4.
template <int G>
struct SweepOccupancy {
  static constexpr int kBlocks = G == 4 ? 3 : 2;
};

// SweepFromCheckerBoardOpt, kernel_functions.cu:2136-2560, G threads per
// pixel, without the prior and propagate-depth paths: jobs with a prior run
// the thread-per-pixel kernel (the launch shape never changes results).
template <int R, int S, int G>
__global__ void __launch_bounds__(kThreads, SweepOccupancy<G>::kBlocks) SweepKernel(const Batch b, int colour) {
  extern __shared__ float smem[];
  __shared__ JobParams sp;
  __shared__ uint64_t mbar;
  int job, blk, iter;
  DecodeBlock(b, b.block_start, blockIdx.x, sp, job, blk, iter);
  const JobParams& p = sp;
  if (iter >= p.num_iterations) return;  // finished job of the batch (block-uniform)
  const float th_mc = p.th_tab[iter];
  const uint64_t skey = StageKey(p.seed, StageSweep(iter, colour));
  constexpr int P = kThreads / G;
  const int bx = b.block_x, rows = P / bx, nb = b.NB;
  const int tw = RefTileW(bx, R), th = rows + 2 * R;
  float* tile = Align128(smem);  // a TMA destination starts on a 128-byte boundary
  float* poses = tile + tw * th;
  SweepSmem sm;
  sm.M = poses + nb * SMVS_POSE_FLOATS;
  sm.HY = sm.M + kMaxHyp * nb * P;
  sm.VW = sm.HY + kMaxHyp * 4 * P;
  sm.PR = sm.VW + nb * P;
  const int col0 = (blk % p.blocks_x) * 2 * bx, row0 = (blk / p.blocks_x) * rows;
  uint32_t tma_uses = 0;
  if (!StageRefTile<R>(b, job, p, tile, row0, col0, rows, poses, &mbar, tma_uses)) return;  // block-uniform
  __syncthreads();
  const int g = threadIdx.x / G, lane = threadIdx.x % G;
  const int row = row0 + g / bx;
  const int col = col0 + 2 * (g % bx) + ((row + colour) & 1);
  if (col >= p.W || row >= p.H) return;  // uniform over the pixel's lanes
  const unsigned gmask = GroupMask<G>();
  const bool leader = lane == 0;
#define M_(h, v) sm.M[((h) * nb + (v)) * P + g]
#define HY_(h, c) sm.HY[((h) * 4 + (c)) * P + g]
#define VW_(v) sm.VW[(v) * P + g]
#define PR_(v) sm.PR[(v) * P + g]
  const int W = p.W, H = p.H, N = p.N;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  Rng r(skey, (uint32_t)pix);
  float depth = p.depth[pix];
  float normal[3] = {p.normal[pix], p.normal[WH + pix], p.normal[2 * WH + pix]};
  const float grad = p.grad[pix];
  const float depth_min = p.depth_min;
  const float depth_max = (float)(1.2 * (double)p.depth_max);  // [quirk] :2213
  const float a1 = fminf(p.rand_a1, (float)(180.0 * 0.0174532925199432));
  const float a2 = fminf(p.rand_a2, (float)(90.0 * 0.0174532925199432));
  const float* iK = p.refiK;
  const float vd[3] = {iK[0] * col + iK[1], iK[2] * row + iK[3], 1.0f};
  const float ivl = rsqrtf(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);

  // Hypothesis list (identical in every lane; lane 0 stores it).
  int ns = 1;
  if (leader) { HY_(0, 0) = normal[0]; HY_(0, 1) = normal[1]; HY_(0, 2) = normal[2]; HY_(0, 3) = depth; }
  if (grad >= 1.0f) {  // :2237-2276
    float nconf[4], O[4];
    int nvalid = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      O[i] = (float)i;
      const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
      if (u < 0 || u >= W || v < 0 || v >= H) { nconf[i] = FLT_MAX; continue; }
      nvalid++;
      nconf[i] = p.conf[(size_t)v * W + u];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3 - i; ++j)
        if (nconf[j] > nconf[j + 1]) {
          float t = nconf[j]; nconf[j] = nconf[j + 1]; nconf[j + 1] = t;
          t = O[j]; O[j] = O[j + 1]; O[j + 1] = t;
        }
    nvalid = min(nvalid, 2);
    for (int i = 0; i < nvalid; ++i) {
      const int idx = (int)O[i];
      const int u = kNeighborOffs[idx][1] + col, v = kNeighborOffs[idx][0] + row;
      const size_t q = (size_t)v * W + u;
      float nn[3] = {p.normal[q], p.normal[WH + q], p.normal[2 * WH + q]};
      CorrectNormal(nn, vd, ivl);
      const float pd = PropagateDepth(p.depth[q], nn, iK, v, u, vd);
      if (leader) { HY_(ns, 0) = nn[0]; HY_(ns, 1) = nn[1]; HY_(ns, 2) = nn[2]; HY_(ns, 3) = pd; }
      ns++;
    }
  }
  for (int k = 0; k < 8; ++k) {  // :2278-2327
    int br = 0, bc = 0;
    float best = FLT_MAX;
#pragma unroll
    for (int s = 0; s < 10; ++s) {
      const int nr = row + kDirSamples[k][2 * s], nc = col + kDirSamples[k][2 * s + 1];
      if (nr < 0 || nr >= H || nc < 0 || nc >= W) continue;
      const float nconf = p.conf[(size_t)nr * W + nc];
      if (best > nconf) { br = nr; bc = nc; best = nconf; }
    }
    if (best < FLT_MAX) {
      const size_t q = (size_t)br * W + bc;
      float nn[3] = {p.normal[q], p.normal[WH + q], p.normal[2 * WH + q]};
      CorrectNormal(nn, vd, ivl);
      const float pd = PropagateDepth(p.depth[q], nn, iK, br, bc, vd);
      if (leader) { HY_(ns, 0) = nn[0]; HY_(ns, 1) = nn[1]; HY_(ns, 2) = nn[2]; HY_(ns, 3) = pd; }
      ns++;
    }
  }
  for (int v = lane; v < N; v += G) M_(0, v) = p.cost[(size_t)v * WH + pix];
  __syncwarp(gmask);

  PixRef pr;
  pr.center = p.ref[pix];
  pr.rsum = p.ref_sum[pix];
  pr.rvar = p.ref_sqsum[pix] - pr.rsum * pr.rsum;
  pr.ws = tw;
  pr.win = tile + (g / bx) * tw + (col - col0) + RefTileShift(R);
  // Two evaluation phases share one call site of the cost code: phase 0 scores
  // the propagated hypotheses 1..ns-1, phase 1 the refinement hypotheses 1..4.
  int h_end = ns;
  for (int phase = 0; phase < 2; ++phase) {
    for (int h = 1; h < h_end; ++h) {
      const float hn[3] = {HY_(h, 0), HY_(h, 1), HY_(h, 2)};
      const float hd = HY_(h, 3);
      for (int v = 0; v < N; ++v) {
        const float c = ViewCost<R, S, G>(p, poses, v, row, col, hd, hn, vd, pr, p.refK, lane, gmask);
        if (leader) M_(h, v) = c;
      }
    }
    __syncwarp(gmask);
    if (phase == 1) break;

    // ACMM view selection, :2364-2427. Per view: its probability (PR), or 0
    // when the view is not good.
    uint32_t flags = 0;
    for (int v = 0; v < N; ++v) {
      unsigned n1 = 0, n2 = 0;
      float pv = 0.f;
      for (int h = 0; h < ns; ++h) {
        const float cst = M_(h, v);
        pv += __expf(-cst * cst * p.inv_beta2);
        n1 += (cst < th_mc);
        n2 += (cst > p.max_mc);
      }
      if ((int)n1 >= p.num_good && (int)n2 <= p.num_bad) flags |= (1u << v);
      else pv = 0.f;
      if (leader) PR_(v) = pv;
    }
    if (flags == 0) return;
    __syncwarp(gmask);
    {  // the CDF, into VW
      float sum = 0.f;
      for (int v = 0; v < N; ++v) sum += PR_(v);
      const float inv = 1.0f / sum;
      float cum = 0.f;
      for (int v = 0; v < N; ++v) {
        cum += PR_(v) * inv;
        if (leader) VW_(v) = cum;
      }
    }
    __syncwarp(gmask);
    // num_samples uniforms draw views: a set of views (random_opt) or a count
    // per view (in PR, written by lane 0 only).
    uint32_t drawn = 0;
    if (leader && !p.random_opt)
      for (int v = 0; v < N; ++v) PR_(v) = 0.f;
    for (int s = 0; s < p.num_samples; ++s) {
      const float rp = r.Uniform() - FLT_EPSILON;
      for (int v = 0; v < N; ++v)
        if (VW_(v) > rp) {
          drawn |= (1u << v);
          if (leader && !p.random_opt) PR_(v) += 1.0f;
          break;
        }
    }
    __syncwarp(gmask);
    float wn = 0.f;
    for (int v = 0; v < N; ++v) wn += p.random_opt ? (float)((drawn >> v) & 1u) : PR_(v);
    if (wn <= 1e-5f) return;
    const float iwn = 1.0f / wn;
    if (leader)
      for (int v = 0; v < N; ++v) VW_(v) = (p.random_opt ? (float)((drawn >> v) & 1u) : PR_(v)) * iwn;
    __syncwarp(gmask);
    uint32_t sel = 0;
    for (int v = 0; v < N; ++v) if (VW_(v) > 0) sel |= (1u << v);
    if (leader) p.view_sel[pix] = sel;
    int mi = -1;
    {
      float m = FLT_MAX;
      for (int h = 0; h < ns; ++h) {
        float cs = 0.f;
        for (int v = 0; v < N; ++v) cs += VW_(v) * M_(h, v);
        if (cs <= m) { m = cs; mi = h; }  // FindMinCost :648-659 ('<=')
      }
    }
    if (mi < 0) return;
    depth = HY_(mi, 3);
    normal[0] = HY_(mi, 0); normal[1] = HY_(mi, 1); normal[2] = HY_(mi, 2);
    __syncwarp(gmask);
    if (mi != 0)
      for (int v = lane; v < N; v += G) M_(0, v) = M_(mi, v);

    // Refinement hypotheses, :2449-2486.
    float nn[3];
    const float pd_min = (1.0f - p.rand_depth_ratio) * depth, pd_max = (1.0f + p.rand_depth_ratio) * depth;
    const float ndepth = r.Uniform() * (pd_max - pd_min) + pd_min;  // PerturbDepth :141-147
    PerturbNormalACMH(normal, nn, a1, a2, r);
    CorrectNormal(nn, vd, ivl);
    const float rdepth = r.Uniform() * (depth_max - depth_min) + depth_min;
    float rn[3];
    RandomNormal(r, vd, rn);
    CorrectNormal(rn, vd, ivl);
    if (leader) {
      HY_(0, 0) = normal[0]; HY_(0, 1) = normal[1]; HY_(0, 2) = normal[2]; HY_(0, 3) = depth;
      HY_(1, 0) = nn[0]; HY_(1, 1) = nn[1]; HY_(1, 2) = nn[2]; HY_(1, 3) = depth;
      HY_(2, 0) = normal[0]; HY_(2, 1) = normal[1]; HY_(2, 2) = normal[2]; HY_(2, 3) = ndepth;
      HY_(3, 0) = rn[0]; HY_(3, 1) = rn[1]; HY_(3, 2) = rn[2]; HY_(3, 3) = depth;
      HY_(4, 0) = normal[0]; HY_(4, 1) = normal[1]; HY_(4, 2) = normal[2]; HY_(4, 3) = rdepth;
    }
    __syncwarp(gmask);
    h_end = 5;
  }
  // :2488-2559: weighted refinement costs, argmin, write back.
  int mi = -1;
  float m = FLT_MAX;
  for (int h = 0; h < 5; ++h) {
    float cs = 0.f;
    for (int v = 0; v < N; ++v) cs += VW_(v) * M_(h, v);
    if (cs <= m) { m = cs; mi = h; }
  }
  if (mi != -1) {
    if (leader) {
      p.conf[pix] = m;
      p.depth[pix] = HY_(mi, 3);
      p.normal[pix] = HY_(mi, 0); p.normal[WH + pix] = HY_(mi, 1); p.normal[2 * WH + pix] = HY_(mi, 2);
    }
    for (int v = lane; v < N; v += G) p.cost[(size_t)v * WH + pix] = M_(mi, v);
  }
#undef M_
#undef HY_
#undef VW_
#undef PR_
}

// LocalOptimization, kernel_functions.cu:2736-2931, G threads per pixel; the
// five hypotheses and their costs live in shared memory.
template <int R, int S, int G>
__global__ void __launch_bounds__(kThreads, SweepOccupancy<G>::kBlocks) LocalOptKernel(const Batch b, int colour) {
  extern __shared__ float smem[];
  __shared__ JobParams sp;
  __shared__ uint64_t mbar;
  int job, blk, iter;
  DecodeBlock(b, b.block_start, blockIdx.x, sp, job, blk, iter);
  const JobParams& p = sp;
  // Iterations > 2 only (patch_match_cuda.cu:861-880); block-uniform.
  if (iter >= p.num_iterations || !p.local_opt || iter <= 2) return;
  const uint64_t skey = StageKey(p.seed, StageLocal(iter, colour));
  constexpr int P = kThreads / G;
  const int bx = b.block_x, rows = P / bx, nb = b.NB;
  const int tw = RefTileW(bx, R), th = rows + 2 * R;
  float* tile = Align128(smem);  // a TMA destination starts on a 128-byte boundary
  float* poses = tile + tw * th;
  float* Ms = poses + nb * SMVS_POSE_FLOATS;  // [5][nb][P]
  const int col0 = (blk % p.blocks_x) * 2 * bx, row0 = (blk / p.blocks_x) * rows;
  uint32_t tma_uses = 0;
  if (!StageRefTile<R>(b, job, p, tile, row0, col0, rows, poses, &mbar, tma_uses)) return;  // block-uniform
  __syncthreads();
  const int g = threadIdx.x / G, lane = threadIdx.x % G;
  const int row = row0 + g / bx;
  const int col = col0 + 2 * (g % bx) + ((row + colour) & 1);
  if (col >= p.W || row >= p.H) return;
  const unsigned gmask = GroupMask<G>();
  const bool leader = lane == 0;
#define M_(h, v) Ms[((h) * nb + (v)) * P + g]
  const int W = p.W, H = p.H, N = p.N;
  const size_t WH = (size_t)W * H;
  const size_t pix = (size_t)row * W + col;
  Rng r(skey, (uint32_t)pix);
  float conf = p.conf[pix];
  float depth = p.depth[pix];
  float normal[3] = {p.normal[pix], p.normal[WH + pix], p.normal[2 * WH + pix]};
  const uint32_t sel = p.view_sel[pix];
  const float a1 = (float)(4.0 * 0.0174532925199432), a2 = (float)(2.0 * 0.0174532925199432);
  const float* iK = p.refiK;
  const float np[3] = {iK[0] * col + iK[1], iK[2] * row + iK[3], 1.0f};
  float m[3] = {normal[0], normal[1], normal[2]};
  float lo = depth, hi = depth;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int u = kNeighborOffs[i][1] + col, v = kNeighborOffs[i][0] + row;
    if (u < 0 || u >= W || v < 0 || v >= H) continue;
    const size_t q = (size_t)v * W + u;
    const float nd = p.depth[q];
    m[0] += p.normal[q]; m[1] += p.normal[WH + q]; m[2] += p.normal[2 * WH + q];
    if (nd <= lo) lo = nd;
    if (nd > hi) hi = nd;
  }
  const float inv_norm = rsqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  m[0] *= inv_norm; m[1] *= inv_norm; m[2] *= inv_norm;
  PixRef pr;
  pr.center = p.ref[pix];
  pr.rsum = p.ref_sum[pix];
  pr.rvar = p.ref_sqsum[pix] - pr.rsum * pr.rsum;
  pr.ws = tw;
  pr.win = tile + (g / bx) * tw + (col - col0) + RefTileShift(R);
  int mi = -1;
  // Rounds 0..4 score five random hypotheses on the selected views; round 5
  // rescores the winner on the unselected views. One call site of the cost code.
  for (int it = 0; it < 6; ++it) {
    float hcur[4];
    if (it < 5) {
      hcur[3] = r.Uniform() * (hi - lo) + lo;
      PerturbNormalACMH(m, hcur, a1, a2, r);
    } else {
      if (mi == -1) break;
      hcur[0] = normal[0]; hcur[1] = normal[1]; hcur[2] = normal[2]; hcur[3] = depth;
    }
    // [quirk] :2916-2919 passes the inverse intrinsics where K is expected when
    // rescoring the unselected views.
    const float* Kg = (it < 5) ? p.refK : p.refiK;
    float mconf = 0.f, mw = 0.f;
    for (int v = 0; v < N; ++v) {
      const bool selected = (sel >> v) & 1u;
      if (selected != (it < 5)) continue;
      const float cost = ViewCost<R, S, G, true>(p, poses, v, row, col, hcur[3], hcur, np, pr, Kg, lane, gmask);
      if (it < 5) {
        if (leader) M_(it, v) = cost;
        mconf += cost;
        mw += 1.f;
      } else if (leader) {
        p.cost[(size_t)v * WH + pix] = cost;
      }
    }
    if (it == 5) break;
    if (mw <= 0.f) return;
    mconf /= mw;
    if (mconf < conf) {
      conf = mconf;
      depth = hcur[3];
      normal[0] = hcur[0]; normal[1] = hcur[1]; normal[2] = hcur[2];
      mi = it;
    }
  }
  __syncwarp(gmask);
  if (mi != -1) {
    if (leader) {
      p.conf[pix] = conf;
      p.depth[pix] = depth;
      p.normal[pix] = normal[0]; p.normal[WH + pix] = normal[1]; p.normal[2 * WH + pix] = normal[2];
    }
    for (int v = lane; v < N; v += G)
      if ((sel >> v) & 1u) p.cost[(size_t)v * WH + pix] = M_(mi, v);
  }
#undef M_
}

static_assert(kSweepHyp == kMaxHyp, "hypotheses per pixel");

template <int R, int S, int G>
cudaError_t LaunchSweepT(const Batch& b, int colour, bool local, cudaStream_t stream) {
  if (b.total_blocks <= 0) return cudaSuccess;
  if (local)
    LocalOptKernel<R, S, G><<<b.total_blocks, kThreads, LocalKernelSmem(R, b.NB, b.block_x, G), stream>>>(b, colour);
  else
    SweepKernel<R, S, G><<<b.total_blocks, kThreads, SweepKernelSmem(R, b.NB, b.block_x, G), stream>>>(b, colour);
  return cudaGetLastError();
}

// Grid of a thread-per-pixel launch: one block per tile, or with b.persistent
// the blocks that fit on the device at once (occupancy x SMs), capped at the
// tile count (and at b.grid_cap when set).
template <typename Kernel>
cudaError_t TilesGrid(Kernel k, const Batch& b, size_t smem, int* grid) {
  *grid = b.total_blocks;
  if (!b.persistent) return cudaSuccess;
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem);
  if (e != cudaSuccess) return e;
  const long long resident = (long long)sms * (per_sm > 0 ? per_sm : 1);
  if (resident < *grid) *grid = (int)resident;
  if (b.grid_cap > 0 && b.grid_cap < *grid) *grid = b.grid_cap;
  return cudaSuccess;
}

template <int R, int S, int NB>
cudaError_t LaunchSweepL(const Batch& b, int colour, bool local, cudaStream_t stream) {
  if (b.total_blocks <= 0) return cudaSuccess;
  const size_t smem = SweepKernelSmem(R, b.NB, b.block_x, 1);
  if (local) {
    LocalOptKernelL<R, S, NB><<<b.total_blocks, kThreads, smem, stream>>>(b, colour);
    return cudaGetLastError();
  }
  int grid = 0;
  const cudaError_t e = TilesGrid(SweepKernelL<R, S, NB>, b, smem, &grid);
  if (e != cudaSuccess) return e;
  SweepKernelL<R, S, NB><<<grid, kThreads, smem, stream>>>(b, colour);
  return cudaGetLastError();
}

template <int R, int S>
cudaError_t LaunchSweepG(const Batch& b, int colour, bool local, cudaStream_t stream) {
  if (b.tpp == 1) {
    if (b.NB <= 8) return LaunchSweepL<R, S, 8>(b, colour, local, stream);
    if (b.NB <= 12) return LaunchSweepL<R, S, 12>(b, colour, local, stream);
    if (b.NB <= 16) return LaunchSweepL<R, S, 16>(b, colour, local, stream);
    return LaunchSweepL<R, S, SMVS_MAX_SRC>(b, colour, local, stream);
  }
  if (b.tpp == 2) return LaunchSweepT<R, S, 2>(b, colour, local, stream);
  if (b.tpp == 4) return LaunchSweepT<R, S, 4>(b, colour, local, stream);
  return cudaErrorInvalidValue;
}

template <int R, int S>
cudaError_t LaunchInitConfT(const Batch& b, cudaStream_t stream) {
  if (b.total_conf_blocks <= 0) return cudaSuccess;
  InitConfKernel<R, S><<<b.total_conf_blocks, dim3(32, kThreads / 32), InitConfKernelSmem(R, b.NB), stream>>>(b);
  return cudaGetLastError();
}

// Let kernel k request up to kMaxDynamicSmem bytes of dynamic shared memory.
template <typename Kernel>
cudaError_t AllowLargeSmem(Kernel k) {
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxDynamicSmem);
}

}  // namespace

// One entry point per window: op 0 = InitConf, 1 = sweep, 2 = local optimisation.
template <int R, int S>
cudaError_t LaunchWindow(const Batch& b, int op, int colour, cudaStream_t stream) {
  if (op == 0) return LaunchInitConfT<R, S>(b, stream);
  return LaunchSweepG<R, S>(b, colour, op == 2, stream);
}

// Opt this window's kernels into large dynamic shared memory (current device).
template <int R, int S>
cudaError_t ConfigureWindow() {
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = AllowLargeSmem(InitConfKernel<R, S>);
  if (e == cudaSuccess) e = AllowLargeSmem(SweepKernel<R, S, 2>);
  if (e == cudaSuccess) e = AllowLargeSmem(SweepKernel<R, S, 4>);
  if (e == cudaSuccess) e = AllowLargeSmem(LocalOptKernel<R, S, 2>);
  if (e == cudaSuccess) e = AllowLargeSmem(LocalOptKernel<R, S, 4>);
  return e;
}

}  // namespace detail
}  // namespace smvs
