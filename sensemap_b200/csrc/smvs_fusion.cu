// smvs_fusion.cu — fusion of depth maps into a point cloud (StereoFusion).
//
// StereoFusion's image loop (SenseMap src/mvs/fusion.cc:1160-1215), FuseImage
// (:1730-1792) and Fuse (:1794-2182) on the GPU, with the results of the
// reference run seed after seed (its fusion threads' row slices taken one
// after another). Compiled with -fmad=false -prec-div=true -prec-sqrt=true
// -ftz=false: the same IEEE single-precision operations, in the same order, as
// the reference's Eigen expressions (see the float helpers below).
//
// Each image is fused in five steps, all in stream order:
//   1. closure: every seed pixel (one warp each, its state in shared memory)
//      collects the pixels its traversal could ever accept — those that pass
//      its reprojection, depth and normal tests, are not fused yet and are
//      reachable from it through such pixels — with the push lists between
//      them in the reference's push order (the seed's record); records over
//      the shared capacity take a thread-per-seed overflow pass;
//   2. claims: for every pixel the seeds whose records hold it; each seed's
//      predecessor on each of its pixels is the latest earlier claimant, and
//      a record keeps its distinct predecessors;
//   3. order: a ticket order in which every predecessor comes first (the seed
//      grid sheared so that key = column + K x row grows along every
//      predecessor pair);
//   4. replay: warps take tickets, wait for their predecessors, read the masks
//      of their record's pixels and find the pixels the reference's traversal
//      fuses — in parallel (a frontier search) where no limit can bind, else
//      by replaying its depth-first traversal (explicit stack, limits) — mark
//      them and release their successors; then they compute the fused point
//      (medians);
//   5. compaction of the points in seed order.
// A traversal only reads or writes the masks of pixels that pass its tests
// (a pixel that fails them is skipped whether or not it is fused), so two
// seeds whose records share no pixel commute, and waiting for every earlier
// claimant of each pixel reproduces the sequential order exactly.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/smvs.h"
#include "../../include/smvs_testing.h"

extern "C" void smvs_internal_set_error(const char* msg);
cudaMemPool_t smvs_internal_device_pool(int device);

namespace {

constexpr int kBlank = 3;              // blank_size (fusion.cc:1757, :1831)
constexpr int kCap = 256;              // record capacity of the closure pass (pixels)
constexpr int kBigCap = 65535;         // record capacity of the overflow pass (u16 indices)
constexpr int kBigBatch = 256;         // overflow seeds per launch
// Scratch bytes of one overflow thread: gid (u32) | derr (f32) | vid (u16) |
// hash slots (u16, from the next 16-byte boundary) | eoff (u32); a multiple of
// 16 so every thread's arrays stay aligned.
constexpr size_t kBigSlotsOff = ((size_t)kBigCap * 10u + 15u) & ~(size_t)15u;
constexpr size_t kBigEoffOff = kBigSlotsOff + 2u * 2u * 65536u;  // eoff (u32, kBigCap + 1)
constexpr size_t kBigStride = (kBigEoffOff + 4u * ((size_t)kBigCap + 1u) + 15u) & ~(size_t)15u;
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr uint32_t kOver = 0xfffffffeu;
constexpr uint32_t kRetry = 0xfffffffdu;  // the record did not fit the pool; built again after it grows
constexpr int kReplayWarps = 4;        // warps per replay block
constexpr int kEdgeSh = 1024;          // push-list entries of a record staged in shared memory
constexpr int kStackSh = 512;          // replay stack entries kept in shared memory per warp
constexpr int kScanItems = 4096;       // items per scan block (256 threads x 16)
constexpr unsigned long long kWaitLimitNs = 20ull * 1000 * 1000 * 1000;  // bounded waits: 20 s
// Test hooks (smvs_test_fusion_waits): a shorter wait bound and a seed whose
// successors are never released, for this thread's next runs.
thread_local unsigned long long t_wait_limit_ns = 0;  // 0: kWaitLimitNs
thread_local long long t_withhold = -1;

// Status bits written by the kernels.
constexpr uint32_t kStTimeout = 1u, kStPool = 2u, kStBad = 4u, kStBig = 8u;

int Fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  smvs_internal_set_error(buf);
  return code;
}

#define FU_CUDA(call)                                                                                      \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return Fail(SMVS_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// One image as the kernels see it.
struct FView {
  float P[12];   // K [R | T], ComposeProjectionMatrix (src/mvs/utils.cc:35-42)
  float iP[12];  // top rows of [P; 0 0 0 1]^-1 (double inverse rounded once)
  int W, H;
  uint32_t base;  // first pixel of the image in the concatenated arrays
  int ov_begin, ov_end;
  int pad;
};

// Per-pixel arrays of all images, concatenated.
struct FMaps {
  const FView* views;
  const int* ov;          // overlapping_images_, concatenated
  const uint8_t* trav;    // per image: used and not yet fused
  const float* D;         // depth
  const float* X;         // inv_P * (col d, row d, d, 1) (fusion.cc:1953-1955)
  const float* Y;
  const float* Z;
  const float* NX;        // inv_R * normal (:1939-1941)
  const float* NY;
  const float* NZ;
  const float* G;         // red-channel gradient (:2007-2021)
  const uint8_t* rgb;     // W*H*3 per image
  uint8_t* mask;          // fused_pixel_masks_
};

struct FConsts {
  float max_sq_reproj;  // max_squared_reproj_error_ (float)
  float min_cos;        // min_cos_normal_error_ (float)
  float derr_thr;       // largest float <= max_depth_error: x > derr_thr <=> (double)x > max_depth_error
  double max_depth_error;
  int with_normal, min_pix, max_pix, max_depth, min_vis;
};

struct FImage {
  int view;
  int cap;  // closure capacity of the fast pass (<= kCap)
  int Rs, Cs, step;
  uint32_t nseeds;
  const int* rows;  // Rs image rows of the seed grid
};

// Record pool of one image. A record (u32 words): cnt, nE, gid[cnt], derr[cnt],
// pred[cnt], eoff[cnt + 1], vid[cnt] (u16), edges[nE bound] (u16).
struct FRecs {
  uint32_t* pool;
  unsigned long long pool_words;
  unsigned long long* used;   // bump cursor (words)
  uint32_t* rec_off;          // per seed: word offset, or kEmpty, kOver, kRetry (no record)
  uint32_t* over_list;        // seeds over kCap
  uint32_t* n_over;
  uint32_t* stats;            // [0] max cnt, [1] max nE, [2] status
};

__host__ __device__ inline uint32_t RecWords(uint32_t cnt, uint32_t ebound) {
  return 2u + 3u * cnt + (cnt + 1u) + (cnt + 1u) / 2u + (ebound + 1u) / 2u;
}

// Bytes of one replay warp's scratch region: stack (u32) | vals (f32) | ids (u32)
// | acc (u16) | flags (u8), rounded to 16.
__host__ __device__ inline size_t ScratchPer(uint32_t cnt, uint32_t stack) {
  return ((size_t)stack * 4u + (size_t)cnt * 11u + 31u) & ~(size_t)15u;
}

// ---- float helpers: the reference's Eigen evaluation order ----------------
// A 3x4 row-major matrix times a Vector4f: one SSE packet product reduced as
// (p0 + p2) + (p1 + p3) (Eigen's predux).
__device__ __forceinline__ float Dot4p(const float* a, float x, float y, float z, float w) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a[0], x), __fmul_rn(a[2], z)), __fadd_rn(__fmul_rn(a[1], y), __fmul_rn(a[3], w)));
}
// P * xyz.homogeneous(): the 3x3 block product plus the last column.
__device__ __forceinline__ float Dot3h(const float* a, float x, float y, float z) {
  return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a[0], x), __fmul_rn(a[1], y)), __fmul_rn(a[2], z)), a[3]);
}
// Vector3f dot product / 3x3 times Vector3f row.
__device__ __forceinline__ float Dot3(float a0, float a1, float a2, float x, float y, float z) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a0, x), __fmul_rn(a1, y)), __fmul_rn(a2, z));
}
__device__ __forceinline__ bool ValidDepth(float d) { return d > 0.0f && isfinite(d); }
// Total order of floats (sign first): the order the medians use.
__device__ __forceinline__ uint32_t FKey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Rounded projection of a point into image u (fusion.cc:2080-2091); false if
// it falls outside the blank border.
__device__ __forceinline__ bool ProjectPixel(const FView& fu, float x, float y, float z, int* row, int* col) {
  const float q0 = Dot3h(fu.P, x, y, z), q1 = Dot3h(fu.P + 4, x, y, z), q2 = Dot3h(fu.P + 8, x, y, z);
  const float uc = roundf(__fdiv_rn(q0, q2)), ur = roundf(__fdiv_rn(q1, q2));
  if (!(uc >= (float)kBlank && ur >= (float)kBlank && uc < (float)(fu.W - kBlank) && ur < (float)(fu.H - kBlank)))
    return false;
  *col = (int)uc;
  *row = (int)ur;
  return true;
}

// ---- point maps -------------------------------------------------------------
__global__ void PointMapKernel(FView v, float R0, float R1, float R2, float R3, float R4, float R5, float R6,
                               float R7, float R8, const float* __restrict__ normal_in, int with_normal,
                               int has_color, float* D, float* X, float* Y, float* Z, float* NX, float* NY,
                               float* NZ, float* G, const uint8_t* __restrict__ rgb) {
  const uint32_t plane = (uint32_t)v.W * (uint32_t)v.H;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < plane; p += gridDim.x * blockDim.x) {
    const int row = (int)(p / (uint32_t)v.W), col = (int)(p - (uint32_t)row * (uint32_t)v.W);
    const uint32_t g = v.base + p;
    const float d = D[g];
    const float cd = __fmul_rn((float)col, d), rd = __fmul_rn((float)row, d);
    X[g] = Dot4p(v.iP, cd, rd, d, 1.0f);
    Y[g] = Dot4p(v.iP + 4, cd, rd, d, 1.0f);
    Z[g] = Dot4p(v.iP + 8, cd, rd, d, 1.0f);
    if (with_normal) {
      const float n0 = normal_in[p], n1 = normal_in[plane + p], n2 = normal_in[2 * plane + p];
      // inv_R = R^T: row i of inv_R is column i of R.
      NX[g] = Dot3(R0, R3, R6, n0, n1, n2);
      NY[g] = Dot3(R1, R4, R7, n0, n1, n2);
      NZ[g] = Dot3(R2, R5, R8, n0, n1, n2);
    }
    float grad = 0.0f;
    if (has_color && col > 1 && col < v.W - 1 && row > 1 && row < v.H - 1) {
      const uint8_t* px = rgb + 3ull * g;
      const float gx = __fdiv_rn((float)((int)px[-3] - (int)px[3]), 255.0f);
      const float gy = __fdiv_rn((float)((int)px[-3 * v.W] - (int)px[3 * v.W]), 255.0f);
      grad = __fsqrt_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)));
    }
    G[g] = grad;
  }
}

// ---- closure ---------------------------------------------------------------
// Membership of a closure under construction: open addressing over the pixel
// index, slots hold node index + 1 (0 = empty).
struct NodeSet {
  uint16_t* slot;
  uint32_t mask;  // table size - 1 (a power of two, at least twice the capacity)
  __device__ __forceinline__ uint32_t Home(uint32_t g) const { return (g * 0x9E3779B1u) >> 7 & mask; }
  __device__ __forceinline__ void Clear() const {
    for (uint32_t i = 0; i <= mask; ++i) slot[i] = 0;
  }
  __device__ __forceinline__ int Find(const uint32_t* gid, uint32_t g) const {
    for (uint32_t h = Home(g);; h = (h + 1) & mask) {
      const uint32_t e = slot[h];
      if (e == 0) return -1;
      if (gid[e - 1] == g) return (int)e - 1;
    }
  }
  __device__ __forceinline__ void Insert(uint32_t g, int idx) const {
    uint32_t h = Home(g);
    while (slot[h] != 0) h = (h + 1) & mask;
    slot[h] = (uint16_t)(idx + 1);
  }
};

// The seed point's projection into image u (column, row, depth), computed once
// per image: a small direct-mapped cache keyed by the image index.
struct SeedProj {
  int u[16];
  float col[16], row[16], z[16];
  __device__ __forceinline__ void Clear() {
    for (int i = 0; i < 16; ++i) u[i] = -1;
  }
  __device__ __forceinline__ void Get(const FView& fu, int ui, float sx, float sy, float sz, float* pc, float* pr,
                                      float* pz) {
    const int h = ui & 15;
    if (u[h] != ui) {
      const float p0 = Dot4p(fu.P, sx, sy, sz, 1.0f), p1 = Dot4p(fu.P + 4, sx, sy, sz, 1.0f),
                  p2 = Dot4p(fu.P + 8, sx, sy, sz, 1.0f);
      u[h] = ui;
      col[h] = __fdiv_rn(p0, p2);
      row[h] = __fdiv_rn(p1, p2);
      z[h] = p2;
    }
    *pc = col[h];
    *pr = row[h];
    *pz = z[h];
  }
};

// The pixels the seed's traversal can accept (see the file comment) into
// gid/vid/derr, and the push lists between them (eoff/edges, in the reference's
// push order: overlapping_images_ of the pixel's image, :2073-2092) while they
// fit `ecap` (*ne > ecap otherwise). Returns the pixel count, 0 when the seed
// itself is fused or has no valid depth, -1 when there are more than `cap`.
__device__ __forceinline__ int BuildClosure(const FMaps& m, const FConsts& c, uint32_t sg, int sv, uint32_t* gid,
                                            uint16_t* vid, float* derr, const NodeSet& set, int cap,
                                            uint32_t* eoff, uint16_t* edges, uint32_t ecap, uint32_t* ne) {
  *ne = 0;
  if (m.mask[sg]) return 0;
  if (!ValidDepth(m.D[sg])) return 0;
  const float sx = m.X[sg], sy = m.Y[sg], sz = m.Z[sg];
  float s0 = 0.f, s1 = 0.f, s2 = 0.f;
  if (c.with_normal) {
    s0 = m.NX[sg];
    s1 = m.NY[sg];
    s2 = m.NZ[sg];
  }
  SeedProj proj;
  proj.Clear();
  set.Clear();
  gid[0] = sg;
  vid[0] = (uint16_t)sv;
  derr[0] = 0.0f;
  set.Insert(sg, 0);
  int cnt = 1;
  uint32_t e = 0;
  for (int i = 0; i < cnt; ++i) {
    eoff[i] = e;
    const uint32_t g = gid[i];
    const FView& fv = m.views[vid[i]];
    const float x = m.X[g], y = m.Y[g], z = m.Z[g];
    for (int k = fv.ov_begin; k < fv.ov_end; ++k) {
      const int u = m.ov[k];
      if (!m.trav[u]) continue;
      const FView& fu = m.views[u];
      int row, col;
      if (!ProjectPixel(fu, x, y, z, &row, &col)) continue;
      const uint32_t q = fu.base + (uint32_t)row * (uint32_t)fu.W + (uint32_t)col;
      if (m.mask[q]) continue;
      int j = set.Find(gid, q);
      if (j < 0) {
        const float dq = m.D[q];
        if (!ValidDepth(dq)) continue;
        // Reprojection and depth error of the seed point in image u (:1893-1912).
        float pc, pr, pz;
        proj.Get(fu, u, sx, sy, sz, &pc, &pr, &pz);
        const float cdiff = __fsub_rn(pc, (float)col), rdiff = __fsub_rn(pr, (float)row);
        const float sq = __fadd_rn(__fmul_rn(cdiff, cdiff), __fmul_rn(rdiff, rdiff));
        if (sq > c.max_sq_reproj) continue;
        const float de = __fdiv_rn(fabsf(__fsub_rn(pz, dq)), dq);
        if (de > c.derr_thr) continue;
        if (c.with_normal && Dot3(s0, s1, s2, m.NX[q], m.NY[q], m.NZ[q]) < c.min_cos) continue;  // :1944-1948
        if (cnt == cap) return -1;
        j = cnt;
        gid[cnt] = q;
        vid[cnt] = (uint16_t)u;
        derr[cnt] = de;
        set.Insert(q, cnt);
        ++cnt;
      }
      if (e < ecap) edges[e] = (uint16_t)j;
      ++e;
    }
  }
  eoff[cnt] = e;
  *ne = e;
  return cnt;
}

// Writes the record of a closure; false when the pool is full. The push lists
// are copied from BuildClosure's, or computed again when they did not fit.
__device__ bool WriteRecord(const FMaps& m, const FRecs& r, uint32_t seed, const uint32_t* gid, const uint16_t* vid,
                            const float* derr, const NodeSet& set, int cnt, const uint32_t* leoff,
                            const uint16_t* ledges, uint32_t lne, bool have_edges) {
  uint32_t ebound = lne;
  if (!have_edges) {
    ebound = 0;
    for (int i = 0; i < cnt; ++i) {
      const FView& fv = m.views[vid[i]];
      ebound += (uint32_t)(fv.ov_end - fv.ov_begin);
    }
  }
  const uint32_t words = RecWords((uint32_t)cnt, ebound);
  const unsigned long long off = atomicAdd(r.used, (unsigned long long)words);
  if (off + words > r.pool_words || off + words > 0xfffffff0ull) {
    atomicOr(&r.stats[2], kStPool);
    r.rec_off[seed] = kRetry;
    return false;
  }
  uint32_t* rec = r.pool + off;
  uint32_t* rg = rec + 2;
  float* rd = reinterpret_cast<float*>(rg + cnt);
  int32_t* rp = reinterpret_cast<int32_t*>(rd + cnt);
  uint32_t* eoff = reinterpret_cast<uint32_t*>(rp + cnt);
  uint16_t* rv = reinterpret_cast<uint16_t*>(eoff + cnt + 1);
  uint16_t* edges = rv + 2 * ((cnt + 1) / 2);
  for (int i = 0; i < cnt; ++i) {
    rg[i] = gid[i];
    rd[i] = derr[i];
    rp[i] = -1;
    rv[i] = vid[i];
  }
  uint32_t e = 0;
  if (have_edges) {
    for (int i = 0; i <= cnt; ++i) eoff[i] = leoff[i];
    for (uint32_t q = 0; q < lne; ++q) edges[q] = ledges[q];
    e = lne;
  } else {
    for (int i = 0; i < cnt; ++i) {
      eoff[i] = e;
      const uint32_t g = gid[i];
      const FView& fv = m.views[vid[i]];
      const float x = m.X[g], y = m.Y[g], z = m.Z[g];
      for (int k = fv.ov_begin; k < fv.ov_end; ++k) {
        const int u = m.ov[k];
        if (!m.trav[u]) continue;
        const FView& fu = m.views[u];
        int row, col;
        if (!ProjectPixel(fu, x, y, z, &row, &col)) continue;
        const int j = set.Find(gid, fu.base + (uint32_t)row * (uint32_t)fu.W + (uint32_t)col);
        if (j < 0) continue;
        if (e < ebound) edges[e] = (uint16_t)j;
        ++e;
      }
    }
    eoff[cnt] = e;
    if (e > ebound) atomicOr(&r.stats[2], kStBad);
  }
  rec[0] = (uint32_t)cnt;
  rec[1] = e;
  r.rec_off[seed] = (uint32_t)off;
  atomicMax(&r.stats[0], (uint32_t)cnt);
  atomicMax(&r.stats[1], e);
  return true;
}

__device__ __forceinline__ uint32_t SeedPixel(const FMaps& m, const FImage& im, uint32_t s) {
  const uint32_t i = s / (uint32_t)im.Cs, j = s - i * (uint32_t)im.Cs;
  const FView& fv = m.views[im.view];
  const uint32_t row = (uint32_t)im.rows[i], col = (uint32_t)(kBlank + (int)j * im.step);
  return fv.base + row * (uint32_t)fv.W + col;
}

constexpr int kSetSlots = 2 * kCap;          // hash slots of the closure pass
constexpr int kBigSetSlots = 2 * 65536;      // hash slots of the overflow pass
constexpr int kEdgeLocal = 2048;             // push-list entries kept by the closure pass

// One warp per seed. The closure under construction lives in shared memory:
// a hash set of its pixels (key = pixel index, value = node index), the
// nodes (pixel, image, depth error, point) and their push lists.
constexpr int kClosureWarps = 4;  // warps (seeds in flight) per closure block
constexpr uint32_t kNoKey = 0xffffffffu;
struct ClosureShared;

struct ClosureShared {
  uint32_t keys[kSetSlots];
  uint32_t gid[kCap];
  uint32_t dpre[kCap + 1];             // push counts of the frontier, prefix-summed
  uint32_t ecnt[kCap];
  uint16_t kidx[kSetSlots];
  uint16_t vid[kCap];
};

// A closure warp's global staging (L2-resident for the whole grid): the push
// lists, their offsets and the depth errors, each written once and read when
// the record is written.
constexpr size_t kStageEoff = 2u * (size_t)kEdgeLocal;                  // u32[kCap + 1]
constexpr size_t kStageDerr = kStageEoff + 4u * ((size_t)kCap + 1u);   // f32[kCap]
constexpr size_t kStageBytes = (kStageDerr + 4u * (size_t)kCap + 15u) & ~(size_t)15u;

// Exclusive prefix sum over a[lo..hi) into out[lo..hi], out[lo] = base.
__device__ __forceinline__ void WarpPrefix(const uint32_t* a, uint32_t* out, int lo, int hi, uint32_t base,
                                           int lane) {
  uint32_t carry = base;
  for (int i0 = lo; i0 < hi; i0 += 32) {
    const int i = i0 + lane;
    const uint32_t x = i < hi ? a[i] : 0u;
    uint32_t incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (i < hi) out[i] = carry + incl - x;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) out[hi] = carry;
  __syncwarp();
}

constexpr size_t kClosureSmem = sizeof(ClosureShared) * kClosureWarps;

// `stage`: kStageBytes per warp of the grid (global memory; tens of MB for the
// whole grid, so they stay in L2).
__global__ void __launch_bounds__(32 * kClosureWarps) ClosureKernel(FMaps m, FConsts c, FImage im, FRecs r,
                                                                    int only_retry, uint8_t* stage) {
  extern __shared__ __align__(16) unsigned char closure_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  ClosureShared& sh = reinterpret_cast<ClosureShared*>(closure_smem)[w];
  uint8_t* const wstage = stage + ((size_t)blockIdx.x * kClosureWarps + w) * kStageBytes;
  uint16_t* const edges = reinterpret_cast<uint16_t*>(wstage);
  uint32_t* const eoff = reinterpret_cast<uint32_t*>(wstage + kStageEoff);
  float* const derr = reinterpret_cast<float*>(wstage + kStageDerr);
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t s = blockIdx.x * kClosureWarps + w; s < im.nseeds; s += gridDim.x * kClosureWarps) {
    if (only_retry && r.rec_off[s] != kRetry) continue;
    const uint32_t sg = SeedPixel(m, im, s);
    if (m.mask[sg] || !ValidDepth(m.D[sg])) {
      if (lane == 0) r.rec_off[s] = kEmpty;
      continue;
    }
    const float sx = m.X[sg], sy = m.Y[sg], sz = m.Z[sg];
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    if (c.with_normal) {
      s0 = m.NX[sg];
      s1 = m.NY[sg];
      s2 = m.NZ[sg];
    }
    for (int h = lane; h < kSetSlots; h += 32) sh.keys[h] = kNoKey;
    __syncwarp();
    if (lane == 0) {
      const uint32_t h = ((sg * 0x9E3779B1u) >> 7) & (uint32_t)(kSetSlots - 1);
      sh.keys[h] = sg;
      sh.kidx[h] = 0;
      sh.gid[0] = sg;
      sh.vid[0] = (uint16_t)im.view;
      derr[0] = 0.0f;
      eoff[0] = 0;
    }
    __syncwarp();
    int cnt = 1, head = 0;
    uint32_t ecur = 0;
    bool over = false;
    // Breadth-first waves: every (frontier pixel, overlapping image) pair is
    // one lane's candidate; pairs run in pixel-major, image order, so the push
    // lists come out in the reference's order.
    while (head < cnt && !over) {
      const int tail = cnt;
      for (int i = head + lane; i < tail; i += 32) {
        const FView& fv = m.views[sh.vid[i]];
        sh.ecnt[i] = (uint32_t)(fv.ov_end - fv.ov_begin);
      }
      __syncwarp();
      WarpPrefix(sh.ecnt, sh.dpre, head, tail, 0u, lane);
      for (int i = head + lane; i < tail; i += 32) sh.ecnt[i] = 0;
      __syncwarp();
      const uint32_t P = sh.dpre[tail];
      for (uint32_t p0 = 0; p0 < P && !over; p0 += 32) {
        const uint32_t p = p0 + lane;
        // 0 none, 1 found/duplicate (read kidx[h] later), 2 owner of a new node
        int kind = 0, i = 0, u = 0;
        uint32_t h = 0, q = 0;
        float de = 0.f;
        if (p < P) {
          int lo = head, hi = tail - 1;  // the frontier pixel whose pushes hold p
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sh.dpre[mid] <= p) lo = mid; else hi = mid - 1;
          }
          i = lo;
          const FView& fv = m.views[sh.vid[i]];
          u = m.ov[fv.ov_begin + (int)(p - sh.dpre[i])];
          int row, col;
          const uint32_t gi = sh.gid[i];
          if (m.trav[u] && ProjectPixel(m.views[u], m.X[gi], m.Y[gi], m.Z[gi], &row, &col)) {
            const FView& fu = m.views[u];
            q = fu.base + (uint32_t)row * (uint32_t)fu.W + (uint32_t)col;
            if (!m.mask[q]) {
              h = ((q * 0x9E3779B1u) >> 7) & (uint32_t)(kSetSlots - 1);
              const volatile uint32_t* vkeys = sh.keys;  // other lanes insert concurrently
              uint32_t key;
              while ((key = vkeys[h]) != kNoKey && key != q) h = (h + 1) & (uint32_t)(kSetSlots - 1);
              if (key == q) {
                kind = 1;
              } else {
                const float dq = m.D[q];
                bool ok = ValidDepth(dq);
                if (ok) {
                  const float p0 = Dot4p(fu.P, sx, sy, sz, 1.0f), p1 = Dot4p(fu.P + 4, sx, sy, sz, 1.0f),
                              p2 = Dot4p(fu.P + 8, sx, sy, sz, 1.0f);
                  const float cdiff = __fsub_rn(__fdiv_rn(p0, p2), (float)col);
                  const float rdiff = __fsub_rn(__fdiv_rn(p1, p2), (float)row);
                  const float sq = __fadd_rn(__fmul_rn(cdiff, cdiff), __fmul_rn(rdiff, rdiff));
                  de = __fdiv_rn(fabsf(__fsub_rn(p2, dq)), dq);
                  ok = !(sq > c.max_sq_reproj) && !(de > c.derr_thr);
                  if (ok && c.with_normal) ok = !(Dot3(s0, s1, s2, m.NX[q], m.NY[q], m.NZ[q]) < c.min_cos);
                }
                if (ok) {  // claim a slot; a lane of this round may hold the same pixel
                  for (;;) {
                    const uint32_t old = atomicCAS(&sh.keys[h], kNoKey, q);
                    if (old == kNoKey) { kind = 2; break; }
                    if (old == q) { kind = 1; break; }
                    h = (h + 1) & (uint32_t)(kSetSlots - 1);
                  }
                }
              }
            }
          }
        }
        __syncwarp();
        const unsigned own = __ballot_sync(0xffffffffu, kind == 2);
        int j = -1;
        if (kind == 2) {
          j = cnt + __popc(own & lt);
          if (j < im.cap) {
            sh.kidx[h] = (uint16_t)j;
            sh.gid[j] = q;
            sh.vid[j] = (uint16_t)u;
            derr[j] = de;
          }
        }
        cnt += __popc(own);
        if (cnt > im.cap) over = true;
        __syncwarp();
        if (kind == 1) j = sh.kidx[h];
        const unsigned val = __ballot_sync(0xffffffffu, j >= 0);
        const uint32_t at = ecur + (uint32_t)__popc(val & lt);
        if (j >= 0 && !over) {
          if (at < (uint32_t)kEdgeLocal) edges[at] = (uint16_t)j;
          atomicAdd(&sh.ecnt[i], 1u);
        }
        ecur += (uint32_t)__popc(val);
        if (ecur > (uint32_t)kEdgeLocal) over = true;
        __syncwarp();
      }
      if (!over) WarpPrefix(sh.ecnt, eoff, head, tail, eoff[head], lane);
      head = tail;
    }
    if (over) {
      if (lane == 0) {
        r.rec_off[s] = kOver;
        const uint32_t k = atomicAdd(r.n_over, 1u);
        r.over_list[k] = s;
      }
      continue;
    }
    // The record, written by the warp.
    const uint32_t ne = ecur;
    const uint32_t words = RecWords((uint32_t)cnt, ne);
    unsigned long long off = 0;
    if (lane == 0) off = atomicAdd(r.used, (unsigned long long)words);
    off = __shfl_sync(0xffffffffu, off, 0);
    if (off + words > r.pool_words || off + words > 0xfffffff0ull) {
      if (lane == 0) {
        atomicOr(&r.stats[2], kStPool);
        r.rec_off[s] = kRetry;
      }
      continue;
    }
    uint32_t* rec = r.pool + off;
    uint32_t* rg = rec + 2;
    float* rd = reinterpret_cast<float*>(rg + cnt);
    int32_t* rpd = reinterpret_cast<int32_t*>(rd + cnt);
    uint32_t* reo = reinterpret_cast<uint32_t*>(rpd + cnt);
    uint16_t* rv = reinterpret_cast<uint16_t*>(reo + cnt + 1);
    uint16_t* redg = rv + 2 * ((cnt + 1) / 2);
    for (int k = lane; k < cnt; k += 32) {
      rg[k] = sh.gid[k];
      rd[k] = derr[k];
      rpd[k] = -1;
      rv[k] = sh.vid[k];
    }
    for (int k = lane; k <= cnt; k += 32) reo[k] = eoff[k];
    for (uint32_t k = lane; k < ne; k += 32) redg[k] = edges[k];
    if (lane == 0) {
      rec[0] = (uint32_t)cnt;
      rec[1] = ne;
      r.rec_off[s] = (uint32_t)off;
      atomicMax(&r.stats[0], (uint32_t)cnt);
      atomicMax(&r.stats[1], ne);
    }
    __syncwarp();
  }
}

// Seeds over the closure pass's capacity, with their scratch in global memory.
__global__ void __launch_bounds__(64) ClosureBigKernel(FMaps m, FConsts c, FImage im, FRecs r, uint32_t first,
                                                       uint32_t count, uint8_t* scratch) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const uint32_t s = r.over_list[first + t];
  uint8_t* base = scratch + (size_t)t * kBigStride;
  uint32_t* gid = reinterpret_cast<uint32_t*>(base);
  float* derr = reinterpret_cast<float*>(base + (size_t)kBigCap * 4u);
  uint16_t* vid = reinterpret_cast<uint16_t*>(base + (size_t)kBigCap * 8u);
  uint16_t* slots = reinterpret_cast<uint16_t*>(base + kBigSlotsOff);
  uint32_t* eoff = reinterpret_cast<uint32_t*>(base + kBigEoffOff);
  const NodeSet set{slots, (uint32_t)kBigSetSlots - 1u};
  uint32_t ne = 0;
  const int cnt = BuildClosure(m, c, SeedPixel(m, im, s), im.view, gid, vid, derr, set, kBigCap, eoff, nullptr, 0,
                               &ne);
  if (cnt <= 0) {  // cannot be empty here; over kBigCap is reported
    if (cnt < 0) atomicOr(&r.stats[2], kStBig);
    r.rec_off[s] = kEmpty;
    return;
  }
  WriteRecord(m, r, s, gid, vid, derr, set, cnt, eoff, nullptr, 0, false);
}

// ---- claims and predecessors ------------------------------------------------
struct RecView {
  uint32_t cnt, ne;
  const uint32_t* gid;
  const float* derr;
  int32_t* pred;
  const uint32_t* eoff;
  const uint16_t* vid;
  const uint16_t* edges;
};

__device__ __forceinline__ RecView OpenRecord(uint32_t* pool, uint32_t off) {
  RecView v;
  uint32_t* rec = pool + off;
  v.cnt = rec[0];
  v.ne = rec[1];
  v.gid = rec + 2;
  v.derr = reinterpret_cast<const float*>(v.gid + v.cnt);
  v.pred = reinterpret_cast<int32_t*>(rec + 2 + 2 * v.cnt);
  v.eoff = rec + 2 + 3 * v.cnt;
  v.vid = reinterpret_cast<const uint16_t*>(v.eoff + v.cnt + 1);
  v.edges = v.vid + 2 * ((v.cnt + 1) / 2);
  return v;
}

// One warp per seed in the claim and predecessor kernels: lanes take the
// record's pixels, so the record is read coalesced and the atomics of a seed
// are in flight together.
__global__ void __launch_bounds__(256) ClaimCountKernel(FRecs r, uint32_t nseeds, uint32_t* claim_cnt) {
  const uint32_t s = (uint32_t)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const uint32_t lane = threadIdx.x & 31;
  if (s >= nseeds) return;
  const uint32_t off = r.rec_off[s];
  if (off >= kRetry) return;
  const RecView v = OpenRecord(r.pool, off);
  for (uint32_t k = lane; k < v.cnt; k += 32) atomicAdd(&claim_cnt[v.gid[k]], 1u);
}

__global__ void __launch_bounds__(256) ClaimFillKernel(FRecs r, uint32_t nseeds, uint32_t* claim_cnt,
                                                       const uint32_t* claim_off, uint32_t* claim_list) {
  const uint32_t s = (uint32_t)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const uint32_t lane = threadIdx.x & 31;
  if (s >= nseeds) return;
  const uint32_t off = r.rec_off[s];
  if (off >= kRetry) return;
  const RecView v = OpenRecord(r.pool, off);
  for (uint32_t k = lane; k < v.cnt; k += 32) {
    const uint32_t g = v.gid[k];
    const uint32_t slot = atomicSub(&claim_cnt[g], 1u) - 1u;  // leaves claim_cnt at zero
    claim_list[claim_off[g] + slot] = s;
  }
}

// Predecessor of each (seed, pixel) and the shear K of the ticket order:
// key(p) < key(s) for every predecessor p of s needs K (i_s - i_p) > j_p - j_s.
// The record's predecessors are written once each at the front of pred[] (the
// replay only waits for them), the rest -1; the first 64 distinct ones are
// recognised as repeats, any beyond that may repeat.
constexpr int kPredSeen = 64;

__global__ void __launch_bounds__(256) PredKernel(FRecs r, uint32_t nseeds, int Cs, const uint32_t* claim_off,
                                                  const uint32_t* claim_list, int* shear) {
  __shared__ int32_t seen_all[8][kPredSeen];
  const uint32_t s = (uint32_t)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const uint32_t lane = threadIdx.x & 31;
  int32_t* seen = seen_all[threadIdx.x >> 5];
  if (s >= nseeds) return;
  const uint32_t off = r.rec_off[s];
  if (off >= kRetry) return;
  RecView v = OpenRecord(r.pool, off);
  const int is = (int)(s / (uint32_t)Cs), js = (int)(s - (uint32_t)is * (uint32_t)Cs);
  const unsigned lt = (1u << lane) - 1u;
  int need = 1;
  uint32_t nu = 0;
  for (uint32_t k0 = 0; k0 < v.cnt; k0 += 32) {
    const uint32_t k = k0 + lane;
    int32_t best = -1;
    if (k < v.cnt) {
      // The latest earlier claimant of this pixel (the list is in no order).
      const uint32_t g = v.gid[k];
      for (uint32_t q = claim_off[g], end = claim_off[g + 1]; q < end; ++q) {
        const uint32_t cl = claim_list[q];
        if (cl < s && (int32_t)cl > best) best = (int32_t)cl;
      }
    }
    bool fresh = best >= 0;
    const uint32_t known = nu < (uint32_t)kPredSeen ? nu : (uint32_t)kPredSeen;
    for (uint32_t t = 0; fresh && t < known; ++t)
      if (seen[t] == best) fresh = false;
    const unsigned same = __match_any_sync(0xffffffffu, best);
    fresh = fresh && (same & lt) == 0;  // the first lane holding this value
    const unsigned nw = __ballot_sync(0xffffffffu, fresh);
    if (fresh) {
      const uint32_t pos = nu + (uint32_t)__popc(nw & lt);
      v.pred[pos] = best;  // pos <= k: this kernel reads no pred[] entry
      if (pos < (uint32_t)kPredSeen) seen[pos] = best;
      const uint32_t p = (uint32_t)best;
      const int ip = (int)(p / (uint32_t)Cs), jp = (int)(p - (uint32_t)ip * (uint32_t)Cs);
      if (ip < is) {
        const int num = jp - js, den = is - ip;
        const int fl = num >= 0 ? num / den : -((-num + den - 1) / den);
        need = max(need, fl + 1);
      }
    }
    nu += (uint32_t)__popc(nw);
    __syncwarp();
  }
  for (uint32_t k = nu + lane; k < v.cnt; k += 32) v.pred[k] = -1;
  for (int o = 16; o > 0; o >>= 1) need = max(need, __shfl_xor_sync(0xffffffffu, need, o));
  if (lane == 0 && need > 1) atomicMax(shear, min(need, Cs));
}

// ---- ticket order ------------------------------------------------------------
__device__ __forceinline__ int KeyRowMin(long long k, int Cs, int K) {
  const long long num = k - Cs + 1;
  return num <= 0 ? 0 : (int)((num + K - 1) / K);
}

__global__ void KeyCountKernel(uint32_t nkeys_cap, int Rs, int Cs, const int* shear, uint32_t* keycnt) {
  const int K = *shear;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nkeys_cap; k += gridDim.x * blockDim.x) {
    const int imin = KeyRowMin(k, Cs, K);
    const int imax = min(Rs - 1, (int)(k / (uint32_t)K));
    keycnt[k] = imax >= imin ? (uint32_t)(imax - imin + 1) : 0u;
  }
}

__global__ void SeqKernel(uint32_t nseeds, int Cs, const int* shear, const uint32_t* keyoff, uint32_t* seq) {
  const int K = *shear;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseeds) return;
  const int i = (int)(s / (uint32_t)Cs), j = (int)(s - (uint32_t)i * (uint32_t)Cs);
  const long long k = (long long)j + (long long)K * i;
  seq[keyoff[k] + (uint32_t)(i - KeyRowMin(k, Cs, K))] = s;
}

// ---- replay -----------------------------------------------------------------
struct FReplay {
  const uint32_t* seq;
  uint32_t nseeds;
  uint32_t* done;
  unsigned int* ticket;
  smvs_fused_point* slot_pts;
  uint32_t* slot_has;
  uint32_t* slot_nvis;
  uint32_t* slot_visoff;
  uint32_t* vis_pool;
  unsigned long long* vis_cursor;
  uint8_t* scratch;           // per-warp scratch for records over the shared budget
  uint32_t scratch_cnt;       // node capacity of a scratch region
  uint32_t scratch_stack;     // stack capacity of a scratch region
  int shared_cnt;             // records up to this many pixels ...
  int shared_stack;           // ... and stack entries replay in shared memory
  uint32_t* level;            // with profiling: dependency depth of each seed (else null)
  uint32_t* chain;            // with profiling: the image's longest dependency chain
  unsigned long long* times;  // with profiling: summed ns [waiting, after the wait until release], seeds
  unsigned long long wait_limit_ns;  // bound of a predecessor wait
  long long withhold;         // test hook: this seed's successors are never released (-1: none, -2: all)
};

struct WarpShared {
  uint32_t stack[kStackSh];
  uint32_t gid[kCap];        // the record, staged before the wait
  uint32_t eoff[kCap + 1];
  float vals[kCap];
  uint32_t ids[kCap];
  uint16_t edges[kEdgeSh];
  uint16_t acc[kCap];
  uint8_t flags[kCap];
  uint32_t bits[kCap / 32];  // reachability search: pixels fused before or reached
  int qtail;
  float med[2];
  int nacc;
};

__device__ __forceinline__ uint32_t LoadAcquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void StoreRelease(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long GlobalTimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Median over vals[0..n) (internal::Median, fusion.cc:47-60) in the total
// order of FKey; ties between equal keys are broken by position.
__device__ float WarpMedian(const float* vals, int n, float* med, int lane) {
  const int mid = n / 2;
  for (int i = lane; i < n; i += 32) {
    const uint32_t ki = FKey(vals[i]);
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const uint32_t kj = FKey(vals[j]);
      rank += (kj < ki || (kj == ki && j < i)) ? 1 : 0;
    }
    if (rank == mid) med[0] = vals[i];
    if ((n & 1) == 0 && rank == mid - 1) med[1] = vals[i];
  }
  __syncwarp();
  const float r = (n & 1) ? med[0] : __fdiv_rn(__fadd_rn(med[0], med[1]), 2.0f);
  __syncwarp();
  return r;
}

// Waits until *flag is set: a short spin, then a growing back-off (fewer loads
// for L2 to serve while most warps wait), bounded in time (status bit on
// timeout).
__device__ __forceinline__ void WaitDone(const uint32_t* flag, uint32_t* stats, unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  unsigned ns = 0;
  for (uint32_t it = 0; LoadAcquire(flag) == 0u; ++it) {
    if (it < 1024) continue;
    if (ns == 0) t0 = GlobalTimer();
    ns = ns < 256 ? ns + 32 : 256;
    __nanosleep(ns);
    if (GlobalTimer() - t0 > limit_ns) {
      atomicOr(&stats[2], kStTimeout);
      return;
    }
  }
}

// The reference's traversal (:1836-2094) on a record, by one lane: LIFO stack
// of (pixel, traversal depth). flags: nonzero = already fused; accepted pixels
// are flagged and listed in acc in the order the reference fuses them. A
// pushed pixel that is already fused would be skipped when popped, so it is
// not pushed. Returns the number accepted.
__device__ int SeqTraversal(uint8_t* __restrict__ flags, uint32_t* __restrict__ stack, uint16_t* __restrict__ acc,
                            const uint32_t* __restrict__ reoff, const uint16_t* __restrict__ redges, int max_pix,
                            int max_depth) {
  int nacc = 0, top = 0;
  if (!flags[0]) stack[top++] = 0u;
  while (top > 0) {
    const uint32_t e = stack[--top];
    const uint32_t k = e & 0xffffu, d = e >> 16;
    if (flags[k]) continue;
    flags[k] = 1;
    acc[nacc++] = (uint16_t)k;
    if (nacc >= max_pix) break;
    if ((int)d + 1 >= max_depth) continue;
    const uint32_t nd = (d + 1 < 0xffffu ? d + 1 : 0xffffu) << 16;
    uint32_t q = reoff[k];
    const uint32_t qe = reoff[k + 1];
    // Four pushes at a time: the loads of a batch overlap (pushes only write
    // the stack, so the flags they read do not change within the batch).
    for (; q + 4 <= qe; q += 4) {
      const uint32_t j0 = redges[q], j1 = redges[q + 1], j2 = redges[q + 2], j3 = redges[q + 3];
      const uint8_t f0 = flags[j0], f1 = flags[j1], f2 = flags[j2], f3 = flags[j3];
      if (!f0) stack[top++] = j0 | nd;
      if (!f1) stack[top++] = j1 | nd;
      if (!f2) stack[top++] = j2 | nd;
      if (!f3) stack[top++] = j3 | nd;
    }
    for (; q < qe; ++q) {
      const uint32_t j = redges[q];
      if (!flags[j]) stack[top++] = j | nd;
    }
  }
  return nacc;
}

__global__ void __launch_bounds__(32 * kReplayWarps) ReplayKernel(FMaps m, FConsts c, FRecs r, FReplay rp) {
  __shared__ WarpShared shm[kReplayWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  WarpShared& sh = shm[w];
  const size_t gw = (size_t)blockIdx.x * kReplayWarps + w;
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(rp.ticket, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= rp.nseeds) break;
    const uint32_t s = rp.seq[t];
    const uint32_t off = r.rec_off[s];
    if (off >= kRetry) continue;  // no record: nothing to fuse, nobody waits for it
    const RecView v = OpenRecord(r.pool, off);
    const int cnt = (int)v.cnt;
    // Storage: the per-pixel arrays in shared memory when the record has at
    // most shared_cnt pixels, the stack when it fits shared_stack entries, and
    // the record itself staged there when it fits; anything larger lives in
    // this warp's global scratch (or is read from the record in place).
    const bool node_sh = cnt <= rp.shared_cnt;
    const bool stack_sh = v.ne + 1 <= (uint32_t)rp.shared_stack;
    if ((!node_sh && (uint32_t)cnt > rp.scratch_cnt) || (!stack_sh && v.ne + 1 > rp.scratch_stack) ||
        ((!node_sh || !stack_sh) && !rp.scratch)) {
      if (lane == 0) {
        atomicOr(&r.stats[2], kStBad);
        StoreRelease(&rp.done[s], 1u);
      }
      continue;
    }
    uint8_t* base = rp.scratch ? rp.scratch + gw * ScratchPer(rp.scratch_cnt, rp.scratch_stack) : nullptr;
    uint32_t* stack = stack_sh ? sh.stack : reinterpret_cast<uint32_t*>(base);
    float* vals;
    uint32_t* ids;
    uint16_t* acc;
    uint8_t* flags;
    if (node_sh) {
      vals = sh.vals;
      ids = sh.ids;
      acc = sh.acc;
      flags = sh.flags;
    } else {
      vals = reinterpret_cast<float*>(base + (size_t)rp.scratch_stack * 4u);
      ids = reinterpret_cast<uint32_t*>(base + (size_t)rp.scratch_stack * 4u + (size_t)rp.scratch_cnt * 4u);
      acc = reinterpret_cast<uint16_t*>(base + (size_t)rp.scratch_stack * 4u + (size_t)rp.scratch_cnt * 8u);
      flags = base + (size_t)rp.scratch_stack * 4u + (size_t)rp.scratch_cnt * 10u;
    }
    const uint32_t* rgid = v.gid;
    const uint32_t* reoff = v.eoff;
    const uint16_t* redges = v.edges;
    if (node_sh) {
      for (int k = lane; k < cnt; k += 32) sh.gid[k] = v.gid[k];
      for (int k = lane; k <= cnt; k += 32) sh.eoff[k] = v.eoff[k];
      rgid = sh.gid;
      reoff = sh.eoff;
      if (v.ne <= (uint32_t)kEdgeSh) {
        for (uint32_t k = lane; k < v.ne; k += 32) sh.edges[k] = v.edges[k];
        redges = sh.edges;
      }
    }
    unsigned long long tw0 = 0;
    if (rp.times) tw0 = GlobalTimer();
    // Wait for the predecessors (every earlier seed that may touch these
    // pixels; the distinct ones come first in pred[]). Lane 0 waits for the
    // latest of them, usually the last to finish; then every lane checks its
    // own entries.
    {
      int32_t latest = -1;
      for (int k = lane; k < cnt; k += 32) {
        const int32_t p = v.pred[k];
        if (p < 0) break;
        latest = max(latest, p);
      }
      for (int o = 16; o > 0; o >>= 1) latest = max(latest, __shfl_xor_sync(0xffffffffu, latest, o));
      if (lane == 0 && latest >= 0) WaitDone(rp.done + latest, r.stats, rp.wait_limit_ns);
      __syncwarp();
      for (int k = lane; k < cnt; k += 32) {
        const int32_t p = v.pred[k];
        if (p < 0) break;
        WaitDone(rp.done + p, r.stats, rp.wait_limit_ns);
      }
    }
    // The acquires above order the predecessors' mask writes before these
    // reads for the whole warp (the barrier orders the lanes).
    __syncwarp();
    unsigned long long tw1 = 0;
    if (rp.times) tw1 = GlobalTimer();
    // Masks are read from L2 (ld.global.cg): other SMs wrote them; a batch of
    // loads is in flight at once.
    {
      int k = lane;
      for (; k + 96 < cnt; k += 128) {
        const uint8_t a0 = __ldcg(m.mask + rgid[k]), a1 = __ldcg(m.mask + rgid[k + 32]),
                      a2 = __ldcg(m.mask + rgid[k + 64]), a3 = __ldcg(m.mask + rgid[k + 96]);
        flags[k] = a0;
        flags[k + 32] = a1;
        flags[k + 64] = a2;
        flags[k + 96] = a3;
      }
      for (; k < cnt; k += 32) flags[k] = __ldcg(m.mask + rgid[k]);
    }
    if (rp.level) {  // profiling: the longest chain of waits ending at this seed
      uint32_t lv = 0;
      for (int k = lane; k < cnt; k += 32) {
        const int32_t p = v.pred[k];
        if (p < 0) break;
        lv = max(lv, *(volatile const uint32_t*)(rp.level + p));
      }
      for (int o = 16; o > 0; o >>= 1) lv = max(lv, __shfl_xor_sync(0xffffffffu, lv, o));
      if (lane == 0) {
        rp.level[s] = lv + 1;
        atomicMax(rp.chain, lv + 1);
      }
    }
    __syncwarp();
    unsigned long long tw_m = 0;
    if (rp.times) tw_m = GlobalTimer();
    // Which record pixels the traversal fuses. Without a binding limit it fuses
    // exactly the pixels reachable from the seed through pixels not fused yet:
    // the warp finds them in parallel (state 0 free, 1 fused before, 2 reached,
    // 3 expanded). The limits cannot bind when at most min(max_num_pixels,
    // max_traversal_depth) pixels are reachable (a pixel's traversal depth is
    // below the number fused); otherwise lane 0 replays the traversal itself.
    bool in_order = false;
    if (node_sh) {
      // Breadth-first search with the record's pixels as bits (fused before,
      // or reached) and the reached pixels queued in acc: each wave expands
      // only the frontier.
      for (int k0 = 0; k0 < cnt; k0 += 32) {
        const int k = k0 + lane;
        const unsigned bal = __ballot_sync(0xffffffffu, k < cnt && flags[k] != 0);
        if (lane == 0) sh.bits[k0 >> 5] = bal;
      }
      __syncwarp();
      if (lane == 0) {
        int t = 0;
        if (!(sh.bits[0] & 1u)) {
          sh.bits[0] |= 1u;
          acc[0] = 0;
          t = 1;
        }
        sh.qtail = t;
      }
      __syncwarp();
      volatile int* vq = &sh.qtail;
      volatile uint32_t* vb = sh.bits;
      int qhead = 0, qt = *vq;
      __syncwarp();
      while (qhead < qt) {
        for (int i = qhead + lane; i < qt; i += 32) {
          const uint32_t k = acc[i];
          for (uint32_t q = reoff[k], qe = reoff[k + 1]; q < qe; ++q) {
            const uint32_t j = redges[q], bit = 1u << (j & 31u);
            if (vb[j >> 5] & bit) continue;
            if (!(atomicOr(&sh.bits[j >> 5], bit) & bit)) acc[atomicAdd(&sh.qtail, 1)] = (uint16_t)j;
          }
        }
        __syncwarp();
        qhead = qt;
        qt = *vq;
        __syncwarp();
      }
      int reach = qt;
      if (rp.times && lane == 0) {
        atomicAdd(rp.times + 3, (unsigned long long)cnt);
        atomicAdd(rp.times + 4, (unsigned long long)reach);
        if (reach > c.max_pix || reach > c.max_depth) atomicAdd(rp.times + 5, 1ull);
      }
      if (reach > c.max_pix || reach > c.max_depth) {  // flags still hold 1 = fused before
        if (lane == 0) reach = SeqTraversal(flags, stack, acc, reoff, redges, c.max_pix, c.max_depth);
        reach = __shfl_sync(0xffffffffu, reach, 0);
        in_order = true;
      }
      if (lane == 0) sh.nacc = reach;
    } else {
      volatile uint8_t* vf = flags;
      if (lane == 0 && vf[0] == 0) vf[0] = 2;
      __syncwarp();
      for (;;) {
        bool any = false;
        for (int k = lane; k < cnt; k += 32) {
          if (vf[k] != 2) continue;
          vf[k] = 3;
          any = true;
          for (uint32_t q = reoff[k], qe = reoff[k + 1]; q < qe; ++q) {
            const uint32_t j = redges[q];
            if (vf[j] == 0) vf[j] = 2;
          }
        }
        __syncwarp();
        if (!__any_sync(0xffffffffu, any)) break;
      }
      int reach = 0;
      for (int k0 = 0; k0 < cnt; k0 += 32) {
        const int k = k0 + lane;
        const bool a = k < cnt && vf[k] == 3;
        const unsigned bal = __ballot_sync(0xffffffffu, a);
        if (a) acc[reach + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)k;
        reach += __popc(bal);
      }
      if (rp.times && lane == 0) {
        atomicAdd(rp.times + 3, (unsigned long long)cnt);
        atomicAdd(rp.times + 4, (unsigned long long)reach);
        if (reach > c.max_pix || reach > c.max_depth) atomicAdd(rp.times + 5, 1ull);
      }
      if (reach > c.max_pix || reach > c.max_depth) {
        for (int k = lane; k < cnt; k += 32) vf[k] = vf[k] == 1 ? 1 : 0;
        __syncwarp();
        if (lane == 0) reach = SeqTraversal(flags, stack, acc, reoff, redges, c.max_pix, c.max_depth);
        reach = __shfl_sync(0xffffffffu, reach, 0);
        in_order = true;
      }
      if (lane == 0) sh.nacc = reach;
    }
    __syncwarp();
    const int n = sh.nacc;
    unsigned long long tw_b = 0;
    if (rp.times) tw_b = GlobalTimer();
    for (int i = lane; i < n; i += 32) *(volatile uint8_t*)(m.mask + rgid[acc[i]]) = 1;
    // Release the successors: the barrier orders every lane's mask writes
    // before lane 0's release store.
    __syncwarp();
    if (lane == 0 && rp.withhold != -2 && (long long)s != rp.withhold) StoreRelease(&rp.done[s], 1u);
    if (rp.times && lane == 0) {
      const unsigned long long tw2 = GlobalTimer();
      atomicAdd(rp.times, tw1 - tw0);
      atomicAdd(rp.times + 1, tw2 - tw1);
      atomicAdd(rp.times + 2, 1ull);
      atomicAdd(rp.times + 6, tw_m - tw1);
      atomicAdd(rp.times + 7, tw_b - tw_m);
      atomicAdd(rp.times + 8, tw2 - tw_b);
    }
    // The fused point (:2098-2180).
    if (n < c.min_pix) continue;
    // Images of the cluster, ascending.
    for (int i = lane; i < n; i += 32) ids[i] = v.vid[acc[i]];
    __syncwarp();
    int nvis = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
      const int i = i0 + lane;
      bool first = false;
      if (i < n) {
        first = true;
        for (int j = 0; j < i; ++j)
          if (ids[j] == ids[i]) {
            first = false;
            break;
          }
      }
      nvis += __popc(__ballot_sync(0xffffffffu, first));
    }
    if (nvis < c.min_vis) continue;
    smvs_fused_point pt;
    memset(&pt, 0, sizeof(pt));
    const float* maps[3] = {m.X, m.Y, m.Z};
    float xyz[3];
    for (int a = 0; a < 3; ++a) {
      for (int i = lane; i < n; i += 32) vals[i] = maps[a][rgid[acc[i]]];
      __syncwarp();
      xyz[a] = WarpMedian(vals, n, sh.med, lane);
    }
    if (!isfinite(xyz[0]) || !isfinite(xyz[1]) || !isfinite(xyz[2])) continue;
    pt.x = xyz[0];
    pt.y = xyz[1];
    pt.z = xyz[2];
    if (c.with_normal) {
      const float* nmaps[3] = {m.NX, m.NY, m.NZ};
      float fn[3];
      for (int a = 0; a < 3; ++a) {
        for (int i = lane; i < n; i += 32) vals[i] = nmaps[a][rgid[acc[i]]];
        __syncwarp();
        fn[a] = WarpMedian(vals, n, sh.med, lane);
      }
      const float norm =
          __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(fn[0], fn[0]), __fmul_rn(fn[1], fn[1])), __fmul_rn(fn[2], fn[2])));
      if (norm < 1.1920928955078125e-07f) continue;  // FLT_EPSILON
      pt.nx = __fdiv_rn(fn[0], norm);
      pt.ny = __fdiv_rn(fn[1], norm);
      pt.nz = __fdiv_rn(fn[2], norm);
    }
    uint8_t rgb[3];
    for (int ch = 0; ch < 3; ++ch) {
      for (int i = lane; i < n; i += 32) vals[i] = (float)m.rgb[3ull * rgid[acc[i]] + ch];
      __syncwarp();
      float med = roundf(WarpMedian(vals, n, sh.med, lane));
      med = med < 255.0f ? med : 255.0f;  // TruncateCast<float, uint8_t>
      med = med > 0.0f ? med : 0.0f;
      rgb[ch] = (uint8_t)med;
    }
    pt.r = rgb[0];
    pt.g = rgb[1];
    pt.b = rgb[2];
    // Mean gradient in traversal order, then the score (:2157-2166). The mean
    // only counts below three images; it needs the pixels in the order the
    // reference fused them, which the parallel search does not give.
    float m_conf = 1.0f;
    if (nvis < 3) {
      if (!in_order) {
        for (int k = lane; k < cnt; k += 32) flags[k] = flags[k] == 1 ? 1 : 0;
        __syncwarp();
        if (lane == 0) SeqTraversal(flags, stack, acc, reoff, redges, c.max_pix, c.max_depth);
        __syncwarp();
      }
      for (int i = lane; i < n; i += 32) vals[i] = m.G[rgid[acc[i]]];
      __syncwarp();
      if (lane == 0) {
        m_conf = 0.0f;
        for (int i = 0; i < n; ++i) m_conf = __fadd_rn(m_conf, vals[i]);
        m_conf = __fdiv_rn(m_conf, (float)n);
      }
      m_conf = __shfl_sync(0xffffffffu, m_conf, 0);
    }
    m_conf = __fsub_rn(1.0f, m_conf);
    __syncwarp();
    for (int i = lane + 1; i < n; i += 32) vals[i - 1] = v.derr[acc[i]];
    __syncwarp();
    const float med_err = WarpMedian(vals, n - 1, sh.med, lane);
    float score = (float)((double)med_err / c.max_depth_error);
    const float mixed = __fadd_rn(__fmul_rn(0.6f, score), __fmul_rn(0.4f, m_conf));
    score = (1.0f < mixed) ? 1.0f : mixed;
    if (!isfinite(score)) continue;
    pt.score = score;
    // Output slot of this seed: the point and its images, ascending.
    uint32_t vbase = 0;
    if (lane == 0) vbase = (uint32_t)atomicAdd(rp.vis_cursor, (unsigned long long)nvis);
    vbase = __shfl_sync(0xffffffffu, vbase, 0);
    for (int i = lane; i < n; i += 32) {
      bool first = true;
      for (int j = 0; j < i; ++j)
        if (ids[j] == ids[i]) {
          first = false;
          break;
        }
      if (!first) continue;
      int rank = 0;  // distinct images below this one
      for (int j = 0; j < n; ++j) {
        if (ids[j] >= ids[i]) continue;
        bool fj = true;
        for (int q = 0; q < j; ++q)
          if (ids[q] == ids[j]) {
            fj = false;
            break;
          }
        rank += fj ? 1 : 0;
      }
      rp.vis_pool[vbase + rank] = ids[i];
    }
    if (lane == 0) {
      rp.slot_pts[s] = pt;
      rp.slot_nvis[s] = (uint32_t)nvis;
      rp.slot_visoff[s] = vbase;
      rp.slot_has[s] = 1u;
    }
    __syncwarp();
  }
}

// ---- scan (exclusive, out[n] = total) ---------------------------------------
__global__ void __launch_bounds__(256) ScanReduceKernel(const uint32_t* in, uint32_t n, uint32_t* sums) {
  __shared__ uint32_t red[256];
  const uint32_t b0 = blockIdx.x * (uint32_t)kScanItems;
  uint32_t acc = 0;
  for (int k = 0; k < kScanItems / 256; ++k) {
    const uint32_t i = b0 + (uint32_t)k * 256u + threadIdx.x;
    if (i < n) acc += in[i];
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int sft = 128; sft > 0; sft >>= 1) {
    if ((int)threadIdx.x < sft) red[threadIdx.x] += red[threadIdx.x + sft];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(1024) ScanSumsKernel(uint32_t* sums, uint32_t nb) {
  __shared__ uint32_t buf[1024];
  uint32_t carry = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += 1024) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t x = i < nb ? sums[i] : 0u;
    buf[threadIdx.x] = x;
    __syncthreads();
    for (int sft = 1; sft < 1024; sft <<= 1) {
      const uint32_t y = (int)threadIdx.x >= sft ? buf[threadIdx.x - sft] : 0u;
      __syncthreads();
      buf[threadIdx.x] += y;
      __syncthreads();
    }
    if (i < nb) sums[i] = carry + buf[threadIdx.x] - x;
    const uint32_t tot = buf[1023];
    __syncthreads();
    carry += tot;
  }
  if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void __launch_bounds__(256) ScanBlockKernel(const uint32_t* in, uint32_t n, const uint32_t* sums,
                                                       uint32_t nb, uint32_t* out) {
  __shared__ uint32_t buf[256];
  const uint32_t b0 = blockIdx.x * (uint32_t)kScanItems;
  uint32_t carry = sums[blockIdx.x];
  for (int k = 0; k < kScanItems / 256; ++k) {
    const uint32_t i = b0 + (uint32_t)k * 256u + threadIdx.x;
    const uint32_t x = i < n ? in[i] : 0u;
    buf[threadIdx.x] = x;
    __syncthreads();
    for (int sft = 1; sft < 256; sft <<= 1) {
      const uint32_t y = (int)threadIdx.x >= sft ? buf[threadIdx.x - sft] : 0u;
      __syncthreads();
      buf[threadIdx.x] += y;
      __syncthreads();
    }
    if (i < n) out[i] = carry + buf[threadIdx.x] - x;
    const uint32_t tot = buf[255];
    __syncthreads();
    carry += tot;
  }
  if (blockIdx.x == nb - 1 && threadIdx.x == 0) out[n] = sums[nb];
}

// ---- per-image bookkeeping and compaction ------------------------------------
__global__ void ImageStartKernel(int* shear, unsigned int* ticket, unsigned long long* rec_used,
                                 unsigned long long* vis_cursor, uint32_t* n_over, uint32_t* stats) {
  *shear = 1;
  *ticket = 0u;
  *rec_used = 0ull;
  *vis_cursor = 0ull;
  *n_over = 0u;
  stats[0] = 0u;
  stats[1] = 0u;
}

__global__ void CompactKernel(uint32_t nseeds, const uint32_t* slot_has, const uint32_t* pt_idx,
                              const uint32_t* vis_idx, const smvs_fused_point* slot_pts, const uint32_t* slot_nvis,
                              const uint32_t* slot_visoff, const uint32_t* vis_pool,
                              const unsigned long long* totals, smvs_fused_point* out_pts, uint64_t* out_visoff,
                              uint32_t* out_vis) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseeds || !slot_has[s]) return;
  const unsigned long long bp = totals[0], bv = totals[1];
  const unsigned long long dst = bp + pt_idx[s], vdst = bv + vis_idx[s];
  out_pts[dst] = slot_pts[s];
  out_visoff[dst] = vdst;
  const uint32_t nv = slot_nvis[s], src = slot_visoff[s];
  for (uint32_t i = 0; i < nv; ++i) out_vis[vdst + i] = vis_pool[src + i];
}

__global__ void AdvanceKernel(unsigned long long* totals, const uint32_t* pt_idx, const uint32_t* vis_idx,
                              uint32_t nseeds, uint64_t* out_visoff) {
  totals[0] += pt_idx[nseeds];
  totals[1] += vis_idx[nseeds];
  out_visoff[totals[0]] = totals[1];
}

}  // namespace

// ---- host object ---------------------------------------------------------------
struct smvs_fusion {
  smvs_fusion_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaMemPool_t pool = nullptr;
  int num_views = 0;
  std::vector<smvs_fusion_view> views;  // sizes and poses (map pointers are not kept)
  std::vector<FView> h_views;
  std::vector<uint8_t> used, fused;
  std::vector<int32_t> ov_off, ov_img;
  std::vector<int> order;
  uint64_t total = 0;  // pixels of all images
  FConsts consts{};
  // Device arrays.
  FView* d_views = nullptr;
  int* d_ov = nullptr;
  uint8_t* d_trav = nullptr;
  float *d_D = nullptr, *d_X = nullptr, *d_Y = nullptr, *d_Z = nullptr, *d_NX = nullptr, *d_NY = nullptr,
        *d_NZ = nullptr, *d_G = nullptr;
  uint8_t* d_rgb = nullptr;
  uint8_t* d_mask = nullptr;
  uint32_t *d_claim_cnt = nullptr, *d_claim_off = nullptr, *d_claim_list = nullptr;
  size_t claim_list_cap = 0;
  uint32_t* d_pool = nullptr;
  size_t pool_words = 0;
  uint32_t *d_rec_off = nullptr, *d_over_list = nullptr, *d_seq = nullptr, *d_done = nullptr;
  uint32_t *d_keycnt = nullptr, *d_keyoff = nullptr;
  size_t key_cap = 0;
  smvs_fused_point* d_slot_pts = nullptr;
  uint32_t *d_slot_has = nullptr, *d_slot_nvis = nullptr, *d_slot_visoff = nullptr;
  uint32_t *d_pt_idx = nullptr, *d_vis_idx = nullptr, *d_vis_pool = nullptr;
  size_t seed_cap = 0;
  uint32_t* d_scan_sums = nullptr;
  size_t scan_sums_cap = 0;
  int* d_rows = nullptr;
  size_t rows_cap = 0;
  uint8_t* d_big_scratch = nullptr;
  uint8_t* d_replay_scratch = nullptr;
  size_t replay_scratch_bytes = 0;
  uint32_t replay_scratch_cnt = 0, replay_scratch_stack = 0;
  // Small device scalars: shear, ticket, n_over, stats[3], counters.
  int* d_shear = nullptr;
  unsigned int* d_ticket = nullptr;
  uint32_t* d_n_over = nullptr;
  uint32_t* d_stats = nullptr;
  unsigned long long* d_used = nullptr;
  unsigned long long* d_vis_cursor = nullptr;
  unsigned long long* d_totals = nullptr;  // [0] points, [1] visibility entries
  // Outputs.
  smvs_fused_point* d_out_pts = nullptr;
  uint64_t* d_out_visoff = nullptr;
  uint32_t* d_out_vis = nullptr;
  uint64_t num_points = 0, num_vis = 0;
  bool ran = false;
  int replay_blocks = 0;
  int closure_blocks = 0;
  uint8_t* d_stage = nullptr;  // the closure warps' global staging
  int cap_closure = kCap, cap_replay = kCap, cap_stack = kStackSh;
  uint32_t* d_level = nullptr;  // profiling: per-seed dependency depth, per-image longest chain
  uint32_t* d_chain = nullptr;
  unsigned long long* d_times = nullptr;  // profiling: per image [wait ns, post-wait ns, seeds]
  size_t level_cap = 0;
  int64_t launches = 0;
  std::vector<int> h_rows;
  bool profiling = false;
  struct Timed { int kind, image; cudaEvent_t a, b; };
  std::vector<double> prof_image_ms;  // 4 per image in fusion order
  std::vector<Timed> timed;
  int prof_count[4] = {0, 0, 0, 0};
  double prof_ms[4] = {0, 0, 0, 0};
};

namespace {

struct ProfScope {
  smvs_fusion* f;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(smvs_fusion* f_, int kind_) : f(f_), kind(kind_) {
    if (!f->profiling) return;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) { a = b = nullptr; return; }
    cudaEventRecord(a, f->stream);
  }
  ~ProfScope() {
    if (!a) return;
    cudaEventRecord(b, f->stream);
    f->timed.push_back({kind, (int)f->order.size(), a, b});
  }
};

void Harvest(smvs_fusion* f) {
  for (auto& t : f->timed) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      f->prof_count[t.kind] += 1;
      f->prof_ms[t.kind] += ms;
      if ((size_t)(4 * t.image + 4) > f->prof_image_ms.size()) f->prof_image_ms.resize(4 * t.image + 4, 0.0);
      f->prof_image_ms[4 * t.image + t.kind] += ms;
    }
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  f->timed.clear();
}

template <typename T>
int Alloc(smvs_fusion* f, T** p, size_t count) {
  const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  cudaError_t err = cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, f->pool, f->stream);
  if (err != cudaSuccess) {
    *p = nullptr;
    return Fail(SMVS_ENOMEM, "fusion: device allocation of %zu bytes: %s", bytes, cudaGetErrorString(err));
  }
  return SMVS_OK;
}

template <typename T>
void Free(smvs_fusion* f, T*& p) {
  if (p) cudaFreeAsync(p, f->stream);
  p = nullptr;
}

void FreeAll(smvs_fusion* f) {
  Harvest(f);
  if (f->pool) {
    Free(f, f->d_views); Free(f, f->d_ov); Free(f, f->d_trav);
    Free(f, f->d_D); Free(f, f->d_X); Free(f, f->d_Y); Free(f, f->d_Z);
    Free(f, f->d_NX); Free(f, f->d_NY); Free(f, f->d_NZ); Free(f, f->d_G);
    Free(f, f->d_rgb); Free(f, f->d_mask);
    Free(f, f->d_claim_cnt); Free(f, f->d_claim_off); Free(f, f->d_claim_list);
    Free(f, f->d_pool); Free(f, f->d_rec_off); Free(f, f->d_over_list); Free(f, f->d_seq); Free(f, f->d_done);
    Free(f, f->d_keycnt); Free(f, f->d_keyoff);
    Free(f, f->d_slot_pts); Free(f, f->d_slot_has); Free(f, f->d_slot_nvis); Free(f, f->d_slot_visoff);
    Free(f, f->d_pt_idx); Free(f, f->d_vis_idx); Free(f, f->d_vis_pool);
    Free(f, f->d_scan_sums); Free(f, f->d_rows); Free(f, f->d_big_scratch); Free(f, f->d_replay_scratch);
    Free(f, f->d_shear); Free(f, f->d_ticket); Free(f, f->d_n_over); Free(f, f->d_stats);
    Free(f, f->d_used); Free(f, f->d_vis_cursor); Free(f, f->d_totals);
    Free(f, f->d_out_pts); Free(f, f->d_out_visoff); Free(f, f->d_out_vis);
    Free(f, f->d_level); Free(f, f->d_chain); Free(f, f->d_stage); Free(f, f->d_times);
  }
  if (f->stream) cudaStreamSynchronize(f->stream);
  if (f->own_stream && f->stream) cudaStreamDestroy(f->stream);
}

// P = K [R | T] in float, Eigen's packet product of a 3x3 and a 3x4 matrix.
void ComposeP(const float K[9], const float R[9], const float T[3], float P[12]) {
  float M[12];
  for (int r = 0; r < 3; ++r) {
    M[4 * r] = R[3 * r];
    M[4 * r + 1] = R[3 * r + 1];
    M[4 * r + 2] = R[3 * r + 2];
    M[4 * r + 3] = T[r];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) {
      volatile float a = K[3 * i] * M[j];
      volatile float b = K[3 * i + 1] * M[4 + j];
      volatile float ab = a + b;
      volatile float c = K[3 * i + 2] * M[8 + j];
      P[4 * i + j] = ab + c;
    }
}

// [P; 0 0 0 1]^-1 in double (adjugate), rounded once.
void ComposeInvP(const float P[12], float iP[12]) {
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

// FindNextImage (fusion.cc:697-727).
int FindNextImage(const smvs_fusion* f, int prev) {
  for (int pass = 0; pass < 2; ++pass)
    for (int32_t k = f->ov_off[prev]; k < f->ov_off[prev + 1]; ++k) {
      const int i = f->ov_img[k];
      if (f->used[i] && !f->fused[i] && (pass == 1 || !f->views[i].is_rig)) return i;
    }
  for (int pass = 0; pass < 2; ++pass)
    for (int i = 0; i < f->num_views; ++i)
      if (f->used[i] && !f->fused[i] && (pass == 1 || !f->views[i].is_rig)) return i;
  return -1;
}

uint32_t Blocks(uint64_t n, int threads) { return (uint32_t)std::max<uint64_t>(1, (n + threads - 1) / threads); }

int EnsureScanSums(smvs_fusion* f, uint64_t n) {
  const size_t nb = (size_t)((n + kScanItems - 1) / kScanItems);
  if (nb + 1 <= f->scan_sums_cap) return SMVS_OK;
  Free(f, f->d_scan_sums);
  f->scan_sums_cap = nb + 1;
  return Alloc(f, &f->d_scan_sums, f->scan_sums_cap);
}

// Exclusive scan of n values into out[0..n], out[n] = total.
int Scan(smvs_fusion* f, const uint32_t* in, uint64_t n, uint32_t* out) {
  if (n == 0) return Fail(SMVS_EINVAL, "fusion: empty scan");
  int st = EnsureScanSums(f, n);
  if (st) return st;
  const uint32_t nb = (uint32_t)((n + kScanItems - 1) / kScanItems);
  ScanReduceKernel<<<nb, 256, 0, f->stream>>>(in, (uint32_t)n, f->d_scan_sums);
  ScanSumsKernel<<<1, 1024, 0, f->stream>>>(f->d_scan_sums, nb);
  ScanBlockKernel<<<nb, 256, 0, f->stream>>>(in, (uint32_t)n, f->d_scan_sums, nb, out);
  f->launches += 3;
  FU_CUDA(cudaGetLastError());
  return SMVS_OK;
}

FMaps Maps(const smvs_fusion* f) {
  FMaps m;
  m.views = f->d_views;
  m.ov = f->d_ov;
  m.trav = f->d_trav;
  m.D = f->d_D;
  m.X = f->d_X;
  m.Y = f->d_Y;
  m.Z = f->d_Z;
  m.NX = f->d_NX;
  m.NY = f->d_NY;
  m.NZ = f->d_NZ;
  m.G = f->d_G;
  m.rgb = f->d_rgb;
  m.mask = f->d_mask;
  return m;
}

FRecs Recs(const smvs_fusion* f) {
  FRecs r;
  r.pool = f->d_pool;
  r.pool_words = f->pool_words;
  r.used = f->d_used;
  r.rec_off = f->d_rec_off;
  r.over_list = f->d_over_list;
  r.n_over = f->d_n_over;
  r.stats = f->d_stats;
  return r;
}

// Per-seed arrays for an image of n seeds.
int EnsureSeeds(smvs_fusion* f, uint64_t n, uint64_t nkeys) {
  int st = SMVS_OK;
  if (n > f->seed_cap) {
    Free(f, f->d_rec_off); Free(f, f->d_over_list); Free(f, f->d_seq); Free(f, f->d_done);
    Free(f, f->d_slot_pts); Free(f, f->d_slot_has); Free(f, f->d_slot_nvis); Free(f, f->d_slot_visoff);
    Free(f, f->d_pt_idx); Free(f, f->d_vis_idx);
    f->seed_cap = n;
    if ((st = Alloc(f, &f->d_rec_off, n)) || (st = Alloc(f, &f->d_over_list, n)) || (st = Alloc(f, &f->d_seq, n)) ||
        (st = Alloc(f, &f->d_done, n)) || (st = Alloc(f, &f->d_slot_pts, n)) || (st = Alloc(f, &f->d_slot_has, n)) ||
        (st = Alloc(f, &f->d_slot_nvis, n)) || (st = Alloc(f, &f->d_slot_visoff, n)) ||
        (st = Alloc(f, &f->d_pt_idx, n + 1)) || (st = Alloc(f, &f->d_vis_idx, n + 1))) {
      f->seed_cap = 0;
      return st;
    }
  }
  if (nkeys > f->key_cap) {
    Free(f, f->d_keycnt); Free(f, f->d_keyoff);
    f->key_cap = nkeys;
    if ((st = Alloc(f, &f->d_keycnt, nkeys)) || (st = Alloc(f, &f->d_keyoff, nkeys + 1))) {
      f->key_cap = 0;
      return st;
    }
  }
  return SMVS_OK;
}

int ReadStats(smvs_fusion* f, uint32_t stats[3], uint32_t* n_over, unsigned long long* used) {
  FU_CUDA(cudaMemcpyAsync(stats, f->d_stats, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, f->stream));
  FU_CUDA(cudaMemcpyAsync(n_over, f->d_n_over, sizeof(uint32_t), cudaMemcpyDeviceToHost, f->stream));
  FU_CUDA(cudaMemcpyAsync(used, f->d_used, sizeof(unsigned long long), cudaMemcpyDeviceToHost, f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  return SMVS_OK;
}

int FuseImage(smvs_fusion* f, int image) {
  const smvs_fusion_view& v = f->views[image];
  const int W = v.width, H = v.height, T = f->opt.num_slices, step = f->opt.step_size;
  // The seed rows of FuseImage's slices (fusion.cc:1733-1764), in order.
  f->h_rows.clear();
  const int hs = (H + T - 1) / T;
  for (int t = 0; t < T; ++t) {
    const int limit = std::min(hs * (t + 1), H);
    const int row_end = std::min(limit, H - kBlank);
    for (int row = std::max(hs * t, kBlank); row < row_end; row += step) f->h_rows.push_back(row);
  }
  const int Rs = (int)f->h_rows.size();
  const int Cs = W - 2 * kBlank > 0 ? (W - 2 * kBlank + step - 1) / step : 0;
  if (Rs == 0 || Cs == 0) {  // no seed pixel: the image is fused all the same
    FU_CUDA(cudaMemsetAsync(f->d_trav + image, 0, 1, f->stream));
    return SMVS_OK;
  }
  const uint64_t nseeds = (uint64_t)Rs * (uint64_t)Cs;
  const uint64_t nkeys = (uint64_t)Cs * (uint64_t)Rs + (uint64_t)Cs;
  int st = EnsureSeeds(f, nseeds, nkeys);
  if (st) return st;
  if ((size_t)Rs > f->rows_cap) {
    Free(f, f->d_rows);
    f->rows_cap = (size_t)Rs;
    if ((st = Alloc(f, &f->d_rows, (size_t)Rs))) { f->rows_cap = 0; return st; }
  }
  FU_CUDA(cudaMemcpyAsync(f->d_rows, f->h_rows.data(), (size_t)Rs * sizeof(int), cudaMemcpyHostToDevice, f->stream));
  FImage im;
  im.view = image;
  im.cap = f->cap_closure;
  im.Rs = Rs;
  im.Cs = Cs;
  im.step = step;
  im.nseeds = (uint32_t)nseeds;
  im.rows = f->d_rows;
  const FMaps m = Maps(f);
  // 1. Closure records (the pool grows until every record fits).
  uint32_t stats[3] = {0, 0, 0}, n_over = 0;
  unsigned long long used = 0;
  ImageStartKernel<<<1, 1, 0, f->stream>>>(f->d_shear, f->d_ticket, f->d_used, f->d_vis_cursor, f->d_n_over,
                                           f->d_stats);
  ++f->launches;
  {
    ProfScope ps(f, SMVS_FUSION_KERNEL_CLOSURE);
    ClosureKernel<<<f->closure_blocks, 32 * kClosureWarps, kClosureSmem, f->stream>>>(m, f->consts, im, Recs(f),
                                                                                         0, f->d_stage);
    ++f->launches;
  }
  FU_CUDA(cudaGetLastError());
  uint32_t big_done = 0;
  for (int attempt = 0;; ++attempt) {
    if ((st = ReadStats(f, stats, &n_over, &used))) return st;
    if (n_over > big_done) {  // seeds over the closure pass's capacity
      if (!f->d_big_scratch && (st = Alloc(f, &f->d_big_scratch, (size_t)kBigBatch * kBigStride))) return st;
      for (uint32_t first = big_done; first < n_over; first += kBigBatch) {
        const uint32_t count = std::min<uint32_t>(kBigBatch, n_over - first);
        ProfScope ps(f, SMVS_FUSION_KERNEL_CLOSURE);
        ClosureBigKernel<<<Blocks(count, 64), 64, 0, f->stream>>>(m, f->consts, im, Recs(f), first, count,
                                                                  f->d_big_scratch);
        ++f->launches;
      }
      FU_CUDA(cudaGetLastError());
      big_done = n_over;
      if ((st = ReadStats(f, stats, &n_over, &used))) return st;
    }
    if (stats[2] & kStBig)
      return Fail(SMVS_EINVAL, "fusion: a seed of image %d reaches more than %d candidate pixels", image, kBigCap);
    if (stats[2] & kStBad) return Fail(SMVS_ECUDA, "fusion: inconsistent cluster record (image %d)", image);
    if (!(stats[2] & kStPool)) break;
    if (attempt >= 8) return Fail(SMVS_ENOMEM, "fusion: record pool cannot grow further");
    // Grow the pool to what this image asked for, plus a margin, keeping the
    // records that fit; only the seeds whose records did not fit run again.
    const size_t old_words = f->pool_words;
    const size_t want = (size_t)std::min<unsigned long long>(used + used / 4 + (1ull << 20), 0xfffffff0ull);
    if (want <= old_words) return Fail(SMVS_ENOMEM, "fusion: record pool limit (16 GB) reached");
    uint32_t* grown = nullptr;
    if ((st = Alloc(f, &grown, want))) return st;
    FU_CUDA(cudaMemcpyAsync(grown, f->d_pool, old_words * sizeof(uint32_t), cudaMemcpyDeviceToDevice, f->stream));
    Free(f, f->d_pool);
    f->d_pool = grown;
    f->pool_words = want;
    const unsigned long long resume = old_words;
    const uint32_t status = stats[2] & ~kStPool;
    FU_CUDA(cudaMemcpyAsync(f->d_used, &resume, sizeof(resume), cudaMemcpyHostToDevice, f->stream));
    FU_CUDA(cudaMemcpyAsync(f->d_stats + 2, &status, sizeof(status), cudaMemcpyHostToDevice, f->stream));
    {
      ProfScope ps(f, SMVS_FUSION_KERNEL_CLOSURE);
      ClosureKernel<<<f->closure_blocks, 32 * kClosureWarps, kClosureSmem, f->stream>>>(m, f->consts, im,
                                                                                           Recs(f), 1, f->d_stage);
      ++f->launches;
    }
    FU_CUDA(cudaGetLastError());
  }
  const uint32_t max_cnt = stats[0], max_ne = stats[1];
  // 2. Claims and predecessors.
  {
    ProfScope ps(f, SMVS_FUSION_KERNEL_ORDER);
    const uint64_t claims = used / 4 + 1;  // a record of cnt pixels takes more than 4 cnt words
    if (claims > f->claim_list_cap) {
      Free(f, f->d_claim_list);
      f->claim_list_cap = (size_t)claims + 1024;
      if ((st = Alloc(f, &f->d_claim_list, f->claim_list_cap))) { f->claim_list_cap = 0; return st; }
    }
    ClaimCountKernel<<<Blocks(32 * nseeds, 256), 256, 0, f->stream>>>(Recs(f), (uint32_t)nseeds, f->d_claim_cnt);
    ++f->launches;
    if ((st = Scan(f, f->d_claim_cnt, f->total, f->d_claim_off))) return st;
    ClaimFillKernel<<<Blocks(32 * nseeds, 256), 256, 0, f->stream>>>(Recs(f), (uint32_t)nseeds, f->d_claim_cnt,
                                                                 f->d_claim_off, f->d_claim_list);
    PredKernel<<<Blocks(32 * nseeds, 256), 256, 0, f->stream>>>(Recs(f), (uint32_t)nseeds, Cs, f->d_claim_off,
                                                           f->d_claim_list, f->d_shear);
    // 3. Ticket order.
    KeyCountKernel<<<Blocks(nkeys, 256), 256, 0, f->stream>>>((uint32_t)nkeys, Rs, Cs, f->d_shear, f->d_keycnt);
    f->launches += 3;
    if ((st = Scan(f, f->d_keycnt, nkeys, f->d_keyoff))) return st;
    SeqKernel<<<Blocks(nseeds, 256), 256, 0, f->stream>>>((uint32_t)nseeds, Cs, f->d_shear, f->d_keyoff, f->d_seq);
    ++f->launches;
    FU_CUDA(cudaGetLastError());
  }
  // 4. Replay.
  if (max_cnt > (uint32_t)f->cap_replay || max_ne + 1 > (uint32_t)f->cap_stack) {
    const uint32_t cap_cnt = std::max<uint32_t>(max_cnt, 1), cap_stack = max_ne + 1;
    const size_t per = ScratchPer(cap_cnt, cap_stack);
    const size_t need = per * (size_t)f->replay_blocks * kReplayWarps;
    if (need > f->replay_scratch_bytes || cap_cnt > f->replay_scratch_cnt || cap_stack > f->replay_scratch_stack) {
      Free(f, f->d_replay_scratch);
      f->replay_scratch_bytes = need;
      if ((st = Alloc(f, &f->d_replay_scratch, need))) { f->replay_scratch_bytes = 0; return st; }
    }
    f->replay_scratch_cnt = cap_cnt;
    f->replay_scratch_stack = cap_stack;
  }
  FU_CUDA(cudaMemsetAsync(f->d_done, 0, nseeds * sizeof(uint32_t), f->stream));
  FU_CUDA(cudaMemsetAsync(f->d_slot_has, 0, nseeds * sizeof(uint32_t), f->stream));
  FU_CUDA(cudaMemsetAsync(f->d_slot_nvis, 0, nseeds * sizeof(uint32_t), f->stream));
  {
    FReplay rp;
    rp.seq = f->d_seq;
    rp.nseeds = (uint32_t)nseeds;
    rp.done = f->d_done;
    rp.ticket = f->d_ticket;
    rp.slot_pts = f->d_slot_pts;
    rp.slot_has = f->d_slot_has;
    rp.slot_nvis = f->d_slot_nvis;
    rp.slot_visoff = f->d_slot_visoff;
    rp.vis_pool = f->d_vis_pool;
    rp.vis_cursor = f->d_vis_cursor;
    rp.scratch = f->d_replay_scratch;
    rp.scratch_cnt = f->d_replay_scratch ? f->replay_scratch_cnt : 0;
    rp.scratch_stack = f->d_replay_scratch ? f->replay_scratch_stack : 0;
    rp.shared_cnt = f->cap_replay;
    rp.shared_stack = f->cap_stack;
    rp.level = nullptr;
    rp.chain = nullptr;
    rp.times = nullptr;
    rp.wait_limit_ns = t_wait_limit_ns ? t_wait_limit_ns : kWaitLimitNs;
    rp.withhold = t_withhold;
    if (f->profiling) {
      if (nseeds > f->level_cap) {
        Free(f, f->d_level);
        f->level_cap = nseeds;
        if ((st = Alloc(f, &f->d_level, nseeds))) { f->level_cap = 0; return st; }
      }
      if (!f->d_chain && (st = Alloc(f, &f->d_chain, 2 * (size_t)f->num_views))) return st;
      const int k = (int)f->order.size();
      FU_CUDA(cudaMemsetAsync(f->d_chain + k, 0, sizeof(uint32_t), f->stream));
      FU_CUDA(cudaMemcpyAsync(f->d_chain + f->num_views + k, f->d_shear, sizeof(uint32_t),
                              cudaMemcpyDeviceToDevice, f->stream));
      rp.level = f->d_level;
      rp.chain = f->d_chain + k;
      if (!f->d_times && (st = Alloc(f, &f->d_times, 9 * (size_t)f->num_views))) return st;
      FU_CUDA(cudaMemsetAsync(f->d_times + 9 * k, 0, 9 * sizeof(unsigned long long), f->stream));
      rp.times = f->d_times + 9 * k;
    }
    ProfScope ps(f, SMVS_FUSION_KERNEL_REPLAY);
    ReplayKernel<<<f->replay_blocks, 32 * kReplayWarps, 0, f->stream>>>(m, f->consts, Recs(f), rp);
    ++f->launches;
    FU_CUDA(cudaGetLastError());
  }
  // 5. Compaction in seed order.
  {
    ProfScope ps(f, SMVS_FUSION_KERNEL_OTHER);
    if ((st = Scan(f, f->d_slot_has, nseeds, f->d_pt_idx))) return st;
    if ((st = Scan(f, f->d_slot_nvis, nseeds, f->d_vis_idx))) return st;
    CompactKernel<<<Blocks(nseeds, 256), 256, 0, f->stream>>>(
        (uint32_t)nseeds, f->d_slot_has, f->d_pt_idx, f->d_vis_idx, f->d_slot_pts, f->d_slot_nvis,
        f->d_slot_visoff, f->d_vis_pool, f->d_totals, f->d_out_pts, f->d_out_visoff, f->d_out_vis);
    AdvanceKernel<<<1, 1, 0, f->stream>>>(f->d_totals, f->d_pt_idx, f->d_vis_idx, (uint32_t)nseeds,
                                          f->d_out_visoff);
    f->launches += 2;
    FU_CUDA(cudaGetLastError());
  }
  // The image is fused: no later traversal enters it.
  FU_CUDA(cudaMemsetAsync(f->d_trav + image, 0, 1, f->stream));
  return SMVS_OK;
}

thread_local int t_cap_closure = 0, t_cap_replay = 0, t_cap_stack = 0;

int CheckStatus(smvs_fusion* f) {
  uint32_t stats[3];
  FU_CUDA(cudaMemcpyAsync(stats, f->d_stats, sizeof(stats), cudaMemcpyDeviceToHost, f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  if (stats[2] & kStTimeout) return Fail(SMVS_ETIMEDOUT, "fusion: a replay wait gave up (predecessor never released)");
  if (stats[2] & kStBad) return Fail(SMVS_ECUDA, "fusion: inconsistent replay state");
  return SMVS_OK;
}

// ---- clean-up passes after the image loop ----------------------------------
// The fused cloud on the host (points, visibility offsets, image indices).
struct HostCloud {
  std::vector<smvs_fused_point> pts;
  std::vector<uint64_t> off;
  std::vector<uint32_t> vis;
};

int Download(smvs_fusion* f, HostCloud& c) {
  c.pts.resize(f->num_points);
  c.off.resize(f->num_points + 1);
  c.vis.resize(f->num_vis);
  if (f->num_points)
    FU_CUDA(cudaMemcpyAsync(c.pts.data(), f->d_out_pts, f->num_points * sizeof(smvs_fused_point),
                            cudaMemcpyDeviceToHost, f->stream));
  FU_CUDA(cudaMemcpyAsync(c.off.data(), f->d_out_visoff, (f->num_points + 1) * sizeof(uint64_t),
                          cudaMemcpyDeviceToHost, f->stream));
  if (f->num_vis)
    FU_CUDA(cudaMemcpyAsync(c.vis.data(), f->d_out_vis, f->num_vis * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  return SMVS_OK;
}

// Keeps the points with keep[i] (order preserved, as the reference's in-place
// compaction loops do) and writes the cloud back to the device arrays, which
// only shrink.
int CompactUpload(smvs_fusion* f, HostCloud& c, const std::vector<uint8_t>& keep, size_t* removed) {
  size_t j = 0, v = 0;
  for (size_t i = 0; i < c.pts.size(); ++i) {
    if (!keep[i]) continue;
    const uint64_t b = c.off[i], e = c.off[i + 1];
    c.pts[j] = c.pts[i];
    c.off[j] = v;
    for (uint64_t k = b; k < e; ++k) c.vis[v++] = c.vis[k];
    ++j;
  }
  c.off[j] = v;
  if (removed) *removed = c.pts.size() - j;
  if (j) FU_CUDA(cudaMemcpyAsync(f->d_out_pts, c.pts.data(), j * sizeof(smvs_fused_point), cudaMemcpyHostToDevice,
                                 f->stream));
  FU_CUDA(cudaMemcpyAsync(f->d_out_visoff, c.off.data(), (j + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice,
                          f->stream));
  if (v) FU_CUDA(cudaMemcpyAsync(f->d_out_vis, c.vis.data(), v * sizeof(uint32_t), cudaMemcpyHostToDevice, f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  f->num_points = j;
  f->num_vis = v;
  return SMVS_OK;
}

// Eigen 3.3's float evaluation of K * (R * X + T) (coefficient-based 3x3
// products reduce as (p0 + p1) + p2), then proj / z rounded half away from
// zero (std::round), as RemoveDuplicatePoints projects (fusion.cc:2216-2219).
void ProjectPoint(const smvs_fusion_view& v, const smvs_fused_point& p, int* u, int* w) {
  const float X[3] = {p.x, p.y, p.z};
  float c[3], q[3];
  for (int r = 0; r < 3; ++r) c[r] = ((v.R[3 * r] * X[0] + v.R[3 * r + 1] * X[1]) + v.R[3 * r + 2] * X[2]) + v.T[r];
  for (int r = 0; r < 3; ++r) q[r] = (v.K[3 * r] * c[0] + v.K[3 * r + 1] * c[1]) + v.K[3 * r + 2] * c[2];
  *u = (int)std::round(q[0] / q[2]);
  *w = (int)std::round(q[1] / q[2]);
}

// Exact k-nearest-neighbour spacing on a uniform grid. Points are bucketed by
// cell (counting sort); each query scans cubes of growing half-width r cells
// around its own cell, keeping the K smallest squared distances (double, the
// coordinate differences squared and summed x, y, z as CGAL's Euclidean
// distance does), and stops once K are known and the K-th lies within r cell
// widths (every point nearer than that is inside the scanned cube; a 1e-9
// relative margin covers the rounding of the cell assignment) or the cube
// covers the grid.
constexpr int kMaxKnn = 64;

struct KnnGrid {
  double minx, miny, minz, h, inv_h;
  int gx, gy, gz;
};

__device__ __forceinline__ int CellCoord(double v, double lo, double inv_h, int g) {
  int c = (int)floor((v - lo) * inv_h);
  return c < 0 ? 0 : (c >= g ? g - 1 : c);
}

__global__ void KnnCountKernel(const smvs_fused_point* __restrict__ pts, uint32_t n, KnnGrid g,
                               uint32_t* __restrict__ cell_of, uint32_t* __restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int cx = CellCoord((double)pts[i].x, g.minx, g.inv_h, g.gx);
  const int cy = CellCoord((double)pts[i].y, g.miny, g.inv_h, g.gy);
  const int cz = CellCoord((double)pts[i].z, g.minz, g.inv_h, g.gz);
  const uint32_t cell = ((uint32_t)cz * g.gy + (uint32_t)cy) * g.gx + (uint32_t)cx;
  cell_of[i] = cell;
  atomicAdd(counts + cell, 1u);
}

__global__ void KnnScatterKernel(uint32_t n, const uint32_t* __restrict__ cell_of, const uint32_t* __restrict__ start,
                                 uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = cell_of[i];
  sorted[start[c] + atomicAdd(cursor + c, 1u)] = i;
}

// ComputeAverageDistance's per-point spacing (patch_match_controller.cc:160-181):
// the mean distance of the query's K = nb_neighbors + 1 nearest points (itself
// included, at distance 0) over K - 1, accumulated nearest first in float with
// each distance added in double.
__global__ void KnnSpacingKernel(const smvs_fused_point* __restrict__ pts, uint32_t n, KnnGrid g,
                                 const uint32_t* __restrict__ start, const uint32_t* __restrict__ sorted, int K,
                                 float* __restrict__ spacing) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double qx = pts[i].x, qy = pts[i].y, qz = pts[i].z;
  const int cx = CellCoord(qx, g.minx, g.inv_h, g.gx);
  const int cy = CellCoord(qy, g.miny, g.inv_h, g.gy);
  const int cz = CellCoord(qz, g.minz, g.inv_h, g.gz);
  double best[kMaxKnn];
  int cnt = 0;
  const int rmax = max(g.gx, max(g.gy, g.gz));
  for (int r = 0; r <= rmax; ++r) {
    // Cells at Chebyshev distance exactly r from the query's cell.
    for (int z = cz - r; z <= cz + r; ++z) {
      if (z < 0 || z >= g.gz) continue;
      for (int y = cy - r; y <= cy + r; ++y) {
        if (y < 0 || y >= g.gy) continue;
        // Inner rows of the shell hold only its two end cells.
        const bool face = (z == cz - r || z == cz + r || y == cy - r || y == cy + r);
        const int step = face ? 1 : 2 * r;
        for (int x = cx - r; x <= cx + r; x += step) {
          if (x < 0 || x >= g.gx) continue;
          const uint32_t cell = ((uint32_t)z * g.gy + (uint32_t)y) * g.gx + (uint32_t)x;
          for (uint32_t k = start[cell]; k < start[cell + 1]; ++k) {
            const smvs_fused_point& p = pts[sorted[k]];
            const double dx = qx - (double)p.x, dy = qy - (double)p.y, dz = qz - (double)p.z;
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
        }
      }
    }
    const double reach = (double)r * g.h * (1.0 - 1e-9);
    if (cnt == K && best[K - 1] <= reach * reach) break;
  }
  float s = 0.0f;
  for (int k = 0; k < cnt; ++k) s = (float)((double)s + sqrt(best[k]));
  if (cnt > 1) s /= (float)(cnt - 1);
  spacing[i] = s;
}

}  // namespace

extern "C" {

int smvs_fusion_options_default(smvs_fusion_options* o) {
  if (!o) return Fail(SMVS_EINVAL, "null options");
  o->step_size = 1;
  o->min_num_pixels = 5;
  o->max_num_pixels = 10000;
  o->min_num_visible_images = 3;
  o->max_traversal_depth = 100;
  o->max_reproj_error = 2.0;
  o->max_depth_error = (double)0.01f;
  o->max_normal_error = 10.0;
  o->with_normal = 1;
  o->num_slices = 1;
  o->gpu_index = 0;
  return SMVS_OK;
}

int smvs_fusion_create(const smvs_fusion_options* opt, const smvs_fusion_view* views, int num_views,
                       const int32_t* overlap_offsets, const int32_t* overlap_images, int memory, void* stream,
                       smvs_fusion** out) {
  if (!opt || !views || num_views < 1 || !overlap_offsets || !out)
    return Fail(SMVS_EINVAL, "fusion: null argument or no images");
  *out = nullptr;
  if (memory != SMVS_MEM_HOST && memory != SMVS_MEM_DEVICE) return Fail(SMVS_EINVAL, "fusion: bad memory kind");
  if (opt->step_size < 1 || opt->min_num_pixels < 2 || opt->max_num_pixels < opt->min_num_pixels ||
      opt->max_traversal_depth < 1 || opt->min_num_visible_images < 0 || opt->num_slices < 1 ||
      !(opt->max_reproj_error >= 0) || !(opt->max_depth_error >= 0) || !(opt->max_normal_error >= 0))
    return Fail(SMVS_EINVAL, "fusion: bad options (min_num_pixels >= 2, max_num_pixels >= min_num_pixels, "
                             "max_traversal_depth > 0, step_size > 0, num_slices > 0, errors >= 0)");
  if (num_views > 65535) return Fail(SMVS_EINVAL, "fusion: more than 65535 images");
  if (overlap_offsets[0] != 0) return Fail(SMVS_EINVAL, "fusion: overlap_offsets[0] must be 0");
  for (int v = 0; v < num_views; ++v) {
    if (overlap_offsets[v + 1] < overlap_offsets[v]) return Fail(SMVS_EINVAL, "fusion: decreasing overlap offsets");
    for (int32_t k = overlap_offsets[v]; k < overlap_offsets[v + 1]; ++k)
      if (!overlap_images || overlap_images[k] < 0 || overlap_images[k] >= num_views)
        return Fail(SMVS_EINVAL, "fusion: overlapping image index out of range");
  }
  uint64_t total = 0;
  for (int v = 0; v < num_views; ++v) {
    const smvs_fusion_view& fv = views[v];
    if (!fv.depth) continue;
    if (fv.width < 1 || fv.height < 1) return Fail(SMVS_EINVAL, "fusion: image %d has no size", v);
    if (opt->with_normal && !fv.normal) return Fail(SMVS_EINVAL, "fusion: image %d has no normal map", v);
    total += (uint64_t)fv.width * (uint64_t)fv.height;
  }
  if (total >= (1ull << 31)) return Fail(SMVS_EINVAL, "fusion: 2^31 pixels or more");
  smvs_fusion* f = new (std::nothrow) smvs_fusion();
  if (!f) return Fail(SMVS_ENOMEM, "fusion: out of host memory");
  f->opt = *opt;
  f->num_views = num_views;
  f->views.assign(views, views + num_views);
  f->ov_off.assign(overlap_offsets, overlap_offsets + num_views + 1);
  f->ov_img.assign(overlap_images ? overlap_images : overlap_offsets,
                   (overlap_images ? overlap_images : overlap_offsets) + overlap_offsets[num_views]);
  f->used.assign(num_views, 0);
  f->fused.assign(num_views, 0);
  f->total = std::max<uint64_t>(total, 1);
  f->device = opt->gpu_index;
  if (t_cap_closure > 0) f->cap_closure = std::min(t_cap_closure, kCap);
  if (t_cap_replay > 0) f->cap_replay = std::min(t_cap_replay, kCap);
  if (t_cap_stack > 0) f->cap_stack = std::min(t_cap_stack, kStackSh);
  auto fail = [&](int st) {
    FreeAll(f);
    delete f;
    return st;
  };
  if (cudaSetDevice(f->device) != cudaSuccess) return fail(Fail(SMVS_ECUDA, "fusion: cannot use GPU %d", f->device));
  if (stream) {
    f->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(Fail(SMVS_ECUDA, "fusion: cannot create a stream"));
    f->own_stream = true;
  }
  f->pool = smvs_internal_device_pool(f->device);
  if (!f->pool) return fail(Fail(SMVS_ECUDA, "fusion: no device memory pool"));
  // Constants (StereoFusion's constructor, fusion.cc:648-663).
  FConsts& c = f->consts;
  c.max_sq_reproj = (float)(opt->max_reproj_error * opt->max_reproj_error);
  c.min_cos = (float)std::cos(opt->max_normal_error * 0.0174532925199432954743716805978692718781530857086181640625);
  float thr = (float)opt->max_depth_error;
  if ((double)thr > opt->max_depth_error) thr = std::nextafter(thr, -INFINITY);
  c.derr_thr = thr;
  c.max_depth_error = opt->max_depth_error;
  c.with_normal = opt->with_normal ? 1 : 0;
  c.min_pix = opt->min_num_pixels;
  c.max_pix = opt->max_num_pixels;
  c.max_depth = opt->max_traversal_depth;
  c.min_vis = opt->min_num_visible_images;
  // Image table.
  f->h_views.resize(num_views);
  uint64_t base = 0;
  for (int v = 0; v < num_views; ++v) {
    FView& hv = f->h_views[v];
    memset(&hv, 0, sizeof(hv));
    ComposeP(views[v].K, views[v].R, views[v].T, hv.P);
    ComposeInvP(hv.P, hv.iP);
    hv.W = views[v].width;
    hv.H = views[v].height;
    hv.base = (uint32_t)base;
    hv.ov_begin = overlap_offsets[v];
    hv.ov_end = overlap_offsets[v + 1];
    f->used[v] = views[v].depth != nullptr;
    if (f->used[v]) base += (uint64_t)hv.W * (uint64_t)hv.H;
    else hv.W = hv.H = 0;
  }
  int st;
  const size_t T = (size_t)f->total;
  const size_t nov = std::max<size_t>((size_t)overlap_offsets[num_views], 1);
  if ((st = Alloc(f, &f->d_views, (size_t)num_views)) || (st = Alloc(f, &f->d_ov, nov)) ||
      (st = Alloc(f, &f->d_trav, (size_t)num_views)) || (st = Alloc(f, &f->d_D, T)) || (st = Alloc(f, &f->d_X, T)) ||
      (st = Alloc(f, &f->d_Y, T)) || (st = Alloc(f, &f->d_Z, T)) || (st = Alloc(f, &f->d_G, T)) ||
      (st = Alloc(f, &f->d_rgb, 3 * T)) || (st = Alloc(f, &f->d_mask, T)) || (st = Alloc(f, &f->d_claim_cnt, T)) ||
      (st = Alloc(f, &f->d_claim_off, T + 1)) || (st = Alloc(f, &f->d_vis_pool, T)) ||
      (st = Alloc(f, &f->d_out_pts, T / 2 + 1)) || (st = Alloc(f, &f->d_out_visoff, T / 2 + 2)) ||
      (st = Alloc(f, &f->d_out_vis, T)) || (st = Alloc(f, &f->d_shear, 1)) || (st = Alloc(f, &f->d_ticket, 1)) ||
      (st = Alloc(f, &f->d_n_over, 1)) || (st = Alloc(f, &f->d_stats, 3)) || (st = Alloc(f, &f->d_used, 1)) ||
      (st = Alloc(f, &f->d_vis_cursor, 1)) || (st = Alloc(f, &f->d_totals, 2)))
    return fail(st);
  if (opt->with_normal &&
      ((st = Alloc(f, &f->d_NX, T)) || (st = Alloc(f, &f->d_NY, T)) || (st = Alloc(f, &f->d_NZ, T))))
    return fail(st);
  // Record pool: 64 words per pixel of the largest image to start with; grows on demand.
  uint64_t max_px = 1;
  for (int v = 0; v < num_views; ++v)
    if (f->used[v]) max_px = std::max<uint64_t>(max_px, (uint64_t)views[v].width * views[v].height);
  // A seed's record holds at most the pixels within the reprojection radius of
  // its point in the image and in each overlapping image (about 16 each for
  // the default 2 pixels), each with one push per overlapping image. Start the
  // pool at that bound for the largest image (within a quarter of the free
  // device memory); it grows if an image needs more.
  int max_deg = 0;
  for (int v = 0; v < num_views; ++v) max_deg = std::max(max_deg, overlap_offsets[v + 1] - overlap_offsets[v]);
  const double radius = std::max(opt->max_reproj_error, 0.5);
  const uint64_t disk = (uint64_t)std::ceil((2.0 * radius + 1.0) * (2.0 * radius + 1.0));
  const uint32_t cnt_est = (uint32_t)std::min<uint64_t>(kCap, disk * (uint64_t)(1 + max_deg));
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
  uint64_t est = max_px * (uint64_t)RecWords(cnt_est, cnt_est * (uint32_t)max_deg);
  est = std::min<uint64_t>(est, std::max<uint64_t>(free_b / 16, max_px * 64ull));
  f->pool_words = (size_t)std::min<uint64_t>(std::max<uint64_t>(est, max_px * 64ull), 0xfffffff0ull);
  if ((st = Alloc(f, &f->d_pool, f->pool_words))) return fail(st);
  auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, f->stream);
  };
  std::vector<uint8_t> trav(f->used.begin(), f->used.end());
  if (up(f->d_views, f->h_views.data(), sizeof(FView) * num_views) != cudaSuccess ||
      (overlap_offsets[num_views] > 0 &&
       up(f->d_ov, overlap_images, sizeof(int32_t) * overlap_offsets[num_views]) != cudaSuccess) ||
      up(f->d_trav, trav.data(), (size_t)num_views) != cudaSuccess ||
      cudaMemsetAsync(f->d_mask, 0, T, f->stream) != cudaSuccess ||
      cudaMemsetAsync(f->d_claim_cnt, 0, T * 4, f->stream) != cudaSuccess ||
      cudaMemsetAsync(f->d_rgb, 0, 3 * T, f->stream) != cudaSuccess ||
      cudaMemsetAsync(f->d_totals, 0, 2 * sizeof(unsigned long long), f->stream) != cudaSuccess ||
      cudaMemsetAsync(f->d_out_visoff, 0, sizeof(uint64_t), f->stream) != cudaSuccess ||
      cudaMemsetAsync(f->d_stats, 0, 3 * sizeof(uint32_t), f->stream) != cudaSuccess)
    return fail(Fail(SMVS_ECUDA, "fusion: upload failed"));
  // Maps and point maps.
  const cudaMemcpyKind kind = memory == SMVS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  for (int v = 0; v < num_views; ++v) {
    if (!f->used[v]) continue;
    const FView& hv = f->h_views[v];
    const size_t plane = (size_t)hv.W * hv.H;
    if (cudaMemcpyAsync(f->d_D + hv.base, views[v].depth, plane * 4, kind, f->stream) != cudaSuccess)
      return fail(Fail(SMVS_ECUDA, "fusion: depth map copy failed"));
    if (views[v].color &&
        cudaMemcpyAsync(f->d_rgb + 3ull * hv.base, views[v].color, plane * 3, kind, f->stream) != cudaSuccess)
      return fail(Fail(SMVS_ECUDA, "fusion: color copy failed"));
    float* d_normal = nullptr;
    if (opt->with_normal) {
      if (memory == SMVS_MEM_HOST) {
        if ((st = Alloc(f, &d_normal, 3 * plane))) return fail(st);
        if (cudaMemcpyAsync(d_normal, views[v].normal, plane * 12, kind, f->stream) != cudaSuccess)
          return fail(Fail(SMVS_ECUDA, "fusion: normal map copy failed"));
      } else {
        d_normal = const_cast<float*>(views[v].normal);
      }
    }
    const float* R = views[v].R;
    PointMapKernel<<<Blocks(plane, 256), 256, 0, f->stream>>>(
        hv, R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7], R[8], d_normal, c.with_normal,
        views[v].color != nullptr, f->d_D, f->d_X, f->d_Y, f->d_Z, f->d_NX, f->d_NY, f->d_NZ, f->d_G, f->d_rgb);
    ++f->launches;
    if (memory == SMVS_MEM_HOST) Free(f, d_normal);
    if (cudaGetLastError() != cudaSuccess) return fail(Fail(SMVS_ECUDA, "fusion: point map launch failed"));
  }
  // The caller's maps are not referenced after this point.
  if (cudaStreamSynchronize(f->stream) != cudaSuccess) return fail(Fail(SMVS_ECUDA, "fusion: upload failed"));
  // Replay grid: every block resident.
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ReplayKernel, 32 * kReplayWarps, 0) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device) != cudaSuccess || per_sm < 1)
    return fail(Fail(SMVS_ECUDA, "fusion: cannot size the replay grid"));
  f->replay_blocks = per_sm * sms;
  if (cudaFuncSetAttribute(ClosureKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClosureSmem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ClosureKernel, 32 * kClosureWarps, kClosureSmem) !=
          cudaSuccess ||
      per_sm < 1)
    return fail(Fail(SMVS_ECUDA, "fusion: cannot size the closure grid"));
  f->closure_blocks = per_sm * sms;
  if ((st = Alloc(f, &f->d_stage, (size_t)f->closure_blocks * kClosureWarps * kStageBytes))) return fail(st);
  *out = f;
  return SMVS_OK;
}

int smvs_fusion_run(smvs_fusion* f) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  if (f->ran) return Fail(SMVS_ESTATE, "fusion: run may be called once");
  if (cudaSetDevice(f->device) != cudaSuccess) return Fail(SMVS_ECUDA, "fusion: cannot use GPU %d", f->device);
  f->ran = true;
  int start = 0;
  for (int i = 0; i < f->num_views; ++i)
    if (!f->views[i].is_rig) {
      start = i;
      break;
    }
  for (int image = start; image >= 0; image = FindNextImage(f, image)) {
    if (!f->used[image]) continue;
    int st = FuseImage(f, image);
    if (st) return st;
    f->fused[image] = 255;
    f->order.push_back(image);
  }
  int st = CheckStatus(f);
  if (st) return st;
  unsigned long long totals[2];
  FU_CUDA(cudaMemcpyAsync(totals, f->d_totals, sizeof(totals), cudaMemcpyDeviceToHost, f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  f->num_points = totals[0];
  f->num_vis = totals[1];
  Harvest(f);
  return SMVS_OK;
}

int smvs_fusion_get_sizes(smvs_fusion* f, size_t* num_points, size_t* num_visibility) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  if (!f->ran) return Fail(SMVS_ESTATE, "fusion: run first");
  if (num_points) *num_points = (size_t)f->num_points;
  if (num_visibility) *num_visibility = (size_t)f->num_vis;
  return SMVS_OK;
}

int smvs_fusion_get_points(smvs_fusion* f, smvs_fused_point* points, uint64_t* vis_offsets, uint32_t* vis_images) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  if (!f->ran) return Fail(SMVS_ESTATE, "fusion: run first");
  if (points && f->num_points)
    FU_CUDA(cudaMemcpyAsync(points, f->d_out_pts, f->num_points * sizeof(smvs_fused_point), cudaMemcpyDefault,
                            f->stream));
  if (vis_offsets)
    FU_CUDA(cudaMemcpyAsync(vis_offsets, f->d_out_visoff, (f->num_points + 1) * sizeof(uint64_t), cudaMemcpyDefault,
                            f->stream));
  if (vis_images && f->num_vis)
    FU_CUDA(cudaMemcpyAsync(vis_images, f->d_out_vis, f->num_vis * sizeof(uint32_t), cudaMemcpyDefault, f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  return SMVS_OK;
}

int smvs_fusion_get_device_points(smvs_fusion* f, const smvs_fused_point** points, const uint64_t** vis_offsets,
                                  const uint32_t** vis_images) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  if (!f->ran) return Fail(SMVS_ESTATE, "fusion: run first");
  if (points) *points = f->d_out_pts;
  if (vis_offsets) *vis_offsets = f->d_out_visoff;
  if (vis_images) *vis_images = f->d_out_vis;
  return SMVS_OK;
}

int smvs_fusion_get_image_order(smvs_fusion* f, int* order, int* count) {
  if (!f || !count) return Fail(SMVS_EINVAL, "null argument");
  *count = (int)f->order.size();
  if (order && !f->order.empty()) memcpy(order, f->order.data(), f->order.size() * sizeof(int));
  return SMVS_OK;
}

int smvs_fusion_get_mask(smvs_fusion* f, int view, uint8_t* out) {
  if (!f || !out) return Fail(SMVS_EINVAL, "null argument");
  if (view < 0 || view >= f->num_views) return Fail(SMVS_EINVAL, "fusion: image %d out of range", view);
  const FView& hv = f->h_views[view];
  const size_t plane = (size_t)f->views[view].width * (size_t)f->views[view].height;
  if (!f->used[view]) {
    memset(out, 0, plane);
    return SMVS_OK;
  }
  FU_CUDA(cudaMemcpyAsync(out, f->d_mask + hv.base, plane, cudaMemcpyDefault, f->stream));
  FU_CUDA(cudaStreamSynchronize(f->stream));
  return SMVS_OK;
}

int smvs_fusion_set_profiling(smvs_fusion* f, int enable) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  f->profiling = enable != 0;
  return SMVS_OK;
}

int smvs_fusion_get_profile(smvs_fusion* f, int kind, int* count, double* total_ms) {
  if (!f || !count || !total_ms || kind < 0 || kind > 3) return Fail(SMVS_EINVAL, "bad profile query");
  Harvest(f);
  *count = f->prof_count[kind];
  *total_ms = f->prof_ms[kind];
  return SMVS_OK;
}

int64_t smvs_fusion_launch_count(smvs_fusion* f) { return f ? f->launches : 0; }

int smvs_test_fusion_chains(smvs_fusion* f, uint32_t* chains, uint32_t* shears, int capacity, int* count) {
  if (!f || !count || capacity < 0 || (capacity > 0 && !chains)) return Fail(SMVS_EINVAL, "null argument");
  if (!f->ran || !f->d_chain) return Fail(SMVS_ESTATE, "fusion chains: run with profiling first");
  const int n = std::min<int>((int)f->order.size(), capacity);
  *count = (int)f->order.size();
  if (n > 0) {
    FU_CUDA(cudaMemcpyAsync(chains, f->d_chain, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost, f->stream));
    if (shears)
      FU_CUDA(cudaMemcpyAsync(shears, f->d_chain + f->num_views, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              f->stream));
    FU_CUDA(cudaStreamSynchronize(f->stream));
  }
  return SMVS_OK;
}

int smvs_test_fusion_image_ms(smvs_fusion* f, double* ms, int capacity, int* count) {
  if (!f || !count || capacity < 0 || (capacity > 0 && !ms)) return Fail(SMVS_EINVAL, "null argument");
  Harvest(f);
  const int n = (int)(f->prof_image_ms.size() / 4);
  *count = n;
  for (int i = 0; i < std::min(n, capacity) * 4; ++i) ms[i] = f->prof_image_ms[i];
  return SMVS_OK;
}

int smvs_test_fusion_replay_times(smvs_fusion* f, double* out, int capacity, int* count) {
  if (!f || !count || capacity < 0 || (capacity > 0 && !out)) return Fail(SMVS_EINVAL, "null argument");
  if (!f->ran || !f->d_times) return Fail(SMVS_ESTATE, "fusion replay times: run with profiling first");
  const int n = (int)f->order.size();
  *count = n;
  std::vector<unsigned long long> t(9 * (size_t)n);
  if (n > 0) {
    FU_CUDA(cudaMemcpyAsync(t.data(), f->d_times, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            f->stream));
    FU_CUDA(cudaStreamSynchronize(f->stream));
  }
  for (int i = 0; i < std::min(n, capacity); ++i) {
    const unsigned long long* ti = t.data() + 9 * i;
    const double seeds = (double)std::max<unsigned long long>(ti[2], 1);
    double* o = out + 9 * i;
    o[0] = (double)ti[0] / seeds / 1000.0;
    o[1] = (double)ti[1] / seeds / 1000.0;
    o[2] = (double)ti[2];
    o[3] = (double)ti[3] / seeds;
    o[4] = (double)ti[4] / seeds;
    o[5] = (double)ti[5];
    o[6] = (double)ti[6] / seeds / 1000.0;
    o[7] = (double)ti[7] / seeds / 1000.0;
    o[8] = (double)ti[8] / seeds / 1000.0;
  }
  return SMVS_OK;
}

int smvs_test_fusion_caps(int closure_cap, int replay_cap, int replay_stack) {
  if (closure_cap < 0 || replay_cap < 0 || replay_stack < 0 || (replay_stack > 0 && replay_stack < 2))
    return Fail(SMVS_EINVAL, "fusion caps: bad values");
  t_cap_closure = closure_cap;
  t_cap_replay = replay_cap;
  t_cap_stack = replay_stack;
  return SMVS_OK;
}

int smvs_test_fusion_waits(double limit_seconds, long long withhold_seed) {
  if (limit_seconds < 0 || withhold_seed < -2) return Fail(SMVS_EINVAL, "fusion waits: bad values");
  t_wait_limit_ns = (unsigned long long)(limit_seconds * 1e9);
  t_withhold = withhold_seed;
  return SMVS_OK;
}

int smvs_fusion_remove_duplicate_points(smvs_fusion* f, size_t* num_removed) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  if (!f->ran) return Fail(SMVS_ESTATE, "fusion: run first");
  if (cudaSetDevice(f->device) != cudaSuccess) return Fail(SMVS_ECUDA, "fusion: cannot use GPU %d", f->device);
  HostCloud c;
  int st = Download(f, c);
  if (st) return st;
  // RemoveDuplicatePoints (fusion.cc:2184-2266): points in fusion order claim
  // the pixel they project to in each of their images; a point meeting an
  // occupant seen by more images is dropped (and looks no further), otherwise
  // it takes the pixel and the occupant is dropped.
  // Occupants as int32 like the reference's Mat<int> (fewer than 2^31 points:
  // the views hold fewer than 2^31 pixels).
  std::vector<std::vector<int32_t>> occ(f->num_views);
  for (int v = 0; v < f->num_views; ++v)
    occ[v].assign((size_t)f->views[v].width * (size_t)f->views[v].height, -1);
  const size_t n = c.pts.size();
  std::vector<uint8_t> removal(n, 0);
  for (size_t i = 0; i < n; ++i) {
    if (removal[i]) continue;
    const uint64_t nvis = c.off[i + 1] - c.off[i];
    for (uint64_t k = c.off[i]; k < c.off[i + 1]; ++k) {
      const int img = (int)c.vis[k];
      const smvs_fusion_view& v = f->views[img];
      int u, w;
      ProjectPoint(v, c.pts[i], &u, &w);
      if (u < 0 || u >= v.width || w < 0 || w >= v.height) continue;
      int32_t& o = occ[img][(size_t)w * v.width + u];
      if (o == -1) {
        o = (int32_t)i;
        continue;
      }
      const uint64_t ovis = c.off[o + 1] - c.off[o];
      if (ovis > nvis) {
        removal[i] = 1;
        break;
      }
      removal[o] = 1;
      o = (int32_t)i;
    }
  }
  std::vector<uint8_t> keep(n);
  for (size_t i = 0; i < n; ++i) keep[i] = !removal[i];
  return CompactUpload(f, c, keep, num_removed);
}

int smvs_fusion_remove_outliers(smvs_fusion* f, int nb_neighbors, double max_spacing_factor, size_t* num_removed) {
  if (!f) return Fail(SMVS_EINVAL, "null fusion");
  if (!f->ran) return Fail(SMVS_ESTATE, "fusion: run first");
  if (nb_neighbors < 1 || nb_neighbors + 1 > kMaxKnn)
    return Fail(SMVS_EINVAL, "fusion: nb_neighbors must be in 1..%d", kMaxKnn - 1);
  if (!(max_spacing_factor > 0)) return Fail(SMVS_EINVAL, "fusion: max_spacing_factor must be > 0");
  if (cudaSetDevice(f->device) != cudaSuccess) return Fail(SMVS_ECUDA, "fusion: cannot use GPU %d", f->device);
  if (num_removed) *num_removed = 0;
  const size_t n = f->num_points;
  if (n == 0) return SMVS_OK;
  if (n >= (1ull << 32) - 1) return Fail(SMVS_EINVAL, "fusion: too many points for the neighbour grid");
  HostCloud c;
  int st = Download(f, c);
  if (st) return st;
  // Grid: about one cell per point over the bounding box (cells of equal
  // side, at least one per axis, at most 2^24 per axis).
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const auto& p : c.pts) {
    const double x[3] = {p.x, p.y, p.z};
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], x[a]); hi[a] = std::max(hi[a], x[a]); }
  }
  if (!(std::isfinite(lo[0]) && std::isfinite(lo[1]) && std::isfinite(lo[2]) && std::isfinite(hi[0]) &&
        std::isfinite(hi[1]) && std::isfinite(hi[2])))
    return Fail(SMVS_EINVAL, "fusion: non-finite point coordinates");
  const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const double emax = std::max(ext[0], std::max(ext[1], ext[2]));
  double vol = 1.0;
  int flat = 0;
  for (int a = 0; a < 3; ++a) {
    if (ext[a] > emax * 1e-6) vol *= ext[a];
    else ++flat;
  }
  double h = emax > 0 ? std::pow(vol / (double)n, 1.0 / (3 - std::min(flat, 2))) : 1.0;
  if (!(h > 0)) h = 1.0;
  KnnGrid g;
  g.minx = lo[0]; g.miny = lo[1]; g.minz = lo[2];
  int dims[3];
  for (;;) {
    for (int a = 0; a < 3; ++a) dims[a] = (int)std::min(16777216.0, std::floor(ext[a] / h) + 1.0);
    if ((double)dims[0] * dims[1] * dims[2] <= 4.0 * (double)n + 64.0) break;
    h *= 1.26;
  }
  g.h = h; g.inv_h = 1.0 / h;
  g.gx = dims[0]; g.gy = dims[1]; g.gz = dims[2];
  const size_t cells = (size_t)g.gx * g.gy * g.gz;
  uint32_t *cell_of = nullptr, *counts = nullptr, *startv = nullptr, *cursor = nullptr, *sorted = nullptr;
  float* spacing = nullptr;
  auto release = [&] {
    Free(f, cell_of); Free(f, counts); Free(f, startv); Free(f, cursor); Free(f, sorted); Free(f, spacing);
  };
  if ((st = Alloc(f, &cell_of, n)) || (st = Alloc(f, &counts, cells)) || (st = Alloc(f, &startv, cells + 1)) ||
      (st = Alloc(f, &cursor, cells)) || (st = Alloc(f, &sorted, n)) || (st = Alloc(f, &spacing, n))) {
    release();
    return st;
  }
  const uint32_t nn = (uint32_t)n;
  const int K = nb_neighbors + 1;
  if (cudaMemsetAsync(counts, 0, cells * sizeof(uint32_t), f->stream) != cudaSuccess ||
      cudaMemsetAsync(cursor, 0, cells * sizeof(uint32_t), f->stream) != cudaSuccess) {
    release();
    return Fail(SMVS_ECUDA, "fusion: clearing the neighbour grid failed");
  }
  KnnCountKernel<<<(nn + 255) / 256, 256, 0, f->stream>>>(f->d_out_pts, nn, g, cell_of, counts);
  st = Scan(f, counts, cells, startv);
  if (!st) {
    KnnScatterKernel<<<(nn + 255) / 256, 256, 0, f->stream>>>(nn, cell_of, startv, cursor, sorted);
    KnnSpacingKernel<<<(nn + 127) / 128, 128, 0, f->stream>>>(f->d_out_pts, nn, g, startv, sorted, K, spacing);
    f->launches += 3;
  }
  std::vector<float> dists(n);
  if (!st && (cudaGetLastError() != cudaSuccess ||
              cudaMemcpyAsync(dists.data(), spacing, n * sizeof(float), cudaMemcpyDeviceToHost, f->stream) !=
                  cudaSuccess ||
              cudaStreamSynchronize(f->stream) != cudaSuccess))
    st = Fail(SMVS_ECUDA, "fusion: neighbour spacing kernels failed");
  release();
  if (st) return st;
  // ComputeAverageDistance's mean (patch_match_controller.cc:184-227): a float
  // sum in point order.
  float average = 0.0f;
  for (size_t i = 0; i < n; ++i) average += dists[i];
  average /= (float)n;
  // RemoveOutliers (fusion.cc:2542-2611): blend each score with its spacing
  // ratio, histogram the scores over 256 bins of [min, max], and drop points
  // in a bin holding under 1 % of the points at or above the 90th cumulative
  // percent.
  if (average > 1e-6) {
    for (size_t i = 0; i < n; ++i) {
      const float factor = (float)((double)dists[i] / (max_spacing_factor * (double)average));
      c.pts[i].score = (float)((double)c.pts[i].score * 0.6 + (double)factor * 0.4);
    }
  }
  float smin = c.pts[0].score, smax = c.pts[0].score;
  for (const auto& p : c.pts) { smin = std::min(smin, p.score); smax = std::max(smax, p.score); }
  const float range = smax - smin;
  // One score for every point (range 0) puts all points in bin 0: none is
  // dropped (the reference divides 0 by 0 there).
  auto bin = [&](float score) -> int {
    if (!(range > 0)) return 0;
    const float gray = (score - smin) / range;
    return (int)(gray * 255);
  };
  std::vector<float> ratios(256, 0.0f), acc(256, 0.0f);
  for (const auto& p : c.pts) ratios[bin(p.score)]++;
  for (int k = 0; k < 256; ++k) ratios[k] /= (float)n;
  float sum = 0.0f;
  for (int k = 0; k < 256; ++k) { sum += ratios[k]; acc[k] = sum; }
  std::vector<uint8_t> keep(n);
  for (size_t i = 0; i < n; ++i) {
    const int b = bin(c.pts[i].score);
    keep[i] = !((double)ratios[b] < 0.01 && (double)acc[b] >= 0.9);
  }
  return CompactUpload(f, c, keep, num_removed);
}

void smvs_fusion_destroy(smvs_fusion* f) {
  if (!f) return;
  cudaSetDevice(f->device);
  FreeAll(f);
  delete f;
}

}  // extern "C"
