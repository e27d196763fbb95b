// smvs_cross_filter.cu — cross-view depth filter and deduplication over a view set.
//
// Replaces CrossFilterCuda (SenseMap src/mvs/patch_match_cuda.h:205-269,
// patch_match_cuda.cu:1111-1710) and its kernels (src/mvs/kernel_functions.cu:
// 3561-3960). The reference packs every view into layered textures padded to
// the largest view, launches one kernel per problem with a device-wide sync
// after each, and for deduplication copies every map back to the host and up
// again. Here:
//   - every view's depth map, decoded normal map, visibility layer, refined
//     map and delta map is a dense W*H region of one HBM buffer per kind
//     (regions start on 128-byte boundaries), read with plain loads;
//   - normals are encoded on the device (NormalMap::Encode, normal_map.cc:
//     159-181) and kept as 4-byte codes; the kernel decodes a code only for
//     the sources that pass the depth tests, with an exact short form of the
//     reference's decode;
//   - Run is one launch over all problems. Its blocks are ordered by image
//     row band first and problem second, so the blocks resident at one time
//     cover the same band of every reference view and read overlapping parts
//     of the source maps from L2; a block stages its problem's parameter block
//     (projection records included) in shared memory, read back with 16-byte
//     loads;
//   - DedupRun keeps the reference's sequential problem order only where two
//     problems touch the same visibility layer: problems are levelled so that
//     any pair with a write/read, read/write or write/write conflict on a layer
//     runs in order, and each level is one launch;
//   - the dedup input of ref_flag views is their refined map in place (no copy);
//   - device memory comes from a per-device stream-ordered pool that keeps
//     freed blocks for the next filter, and no call waits for the GPU except
//     the getters (which copy to the host) and set-up from host memory.
// The unit is compiled without FMA contraction and with IEEE division and
// square root; the fused multiply-adds it performs are written out (fmaf), in
// the same places as in the CPU oracle, so the two agree bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/smvs.h"

extern "C" void smvs_internal_set_error(const char* msg);
void smvs_internal_pose_record(const smvs_view* ref, const smvs_view* src, float* out43);

namespace {

constexpr uint32_t kVisKeep = 0x80000000u;
constexpr int kBlockX = 32, kBlockY = 8, kThreads = kBlockX * kBlockY;
constexpr int kRec = 36;  // per-source record: P (12) | P^-1 (12) | R (9) + 3 pad

int Fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  smvs_internal_set_error(buf);
  return code;
}

#define CF_CUDA(call)                                                                                      \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return Fail(SMVS_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// One source view of a problem as the kernels see it.
struct CfSrc {
  const float* depth;   // depth map (run: input map; dedup: the view's dedup input)
  const uint32_t* aux;  // run: normal codes; dedup: visibility layer
  int width, height, ref_flag, pad;
};

// Parameter block of one problem. Staged into shared memory up to the
// records of its num_src sources.
struct alignas(16) CfJob {
  int width, height, num_src, min_cons;
  int blocks_x, pad0, pad1, pad2;
  float refK[4];    // fx cx fy cy of the reference view
  float refiK[4];   // 1/fx, -cx/fx, 1/fy, -cy/fy (InitTransforms :1330-1334)
  const float* depth;     // reference map
  const uint32_t* code;   // run: reference normal codes
  uint32_t* vis;          // dedup: reference visibility layer
  float* out;             // run: refined map; dedup: delta map
  CfSrc src[SMVS_CROSS_MAX_SRC];
  alignas(16) float rec[SMVS_CROSS_MAX_SRC][kRec];
};
static_assert(sizeof(CfJob) % 16 == 0, "CfJob is staged in 16-byte units");
static_assert(offsetof(CfJob, rec) % 16 == 0, "records are read with 16-byte loads");

// Thresholds shared by every problem (options of the set).
struct CfConsts {
  float fmax_err;      // filter_geom_consistency_max_cost
  float thr;           // depth_diff_threshold
  float thr2;          // its square
  float max_view_cos;  // cosf(DEG2RAD(100))
  float max_cos;       // cosf(DEG2RAD(max_normal_error))
};

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
// Copies the job's header, source table and the records it uses.
__device__ __forceinline__ void StageJob(CfJob* sj, const CfJob* __restrict__ gj) {
  const int ns = __ldg(&gj->num_src);
  const int n16 = (int)((offsetof(CfJob, rec) + (size_t)ns * kRec * sizeof(float) + 15) / 16);
  const int4* g = reinterpret_cast<const int4*>(gj);
  int4* s = reinterpret_cast<int4*>(sj);
  for (int i = threadIdx.x; i < n16; i += kThreads) s[i] = __ldg(g + i);
}

// a . x + t and a . b with explicit fused multiply-adds (the oracle's order).
__device__ __forceinline__ float Affine3(float a0, float a1, float a2, const float x[3], float t) {
  return fmaf(a0, x[0], fmaf(a1, x[1], fmaf(a2, x[2], t)));
}
__device__ __forceinline__ float Dot3(const float a[3], const float b[3]) {
  return fmaf(a[0], b[0], fmaf(a[1], b[1], a[2] * b[2]));
}

// NormalMap::Encode (normal_map.cc:159-181).
__device__ __forceinline__ uint32_t Encode(float n0, float n1, float n2) {
  const float s0 = (float)((1 - n0) * 0.5);
  const float m = 1.0f / sqrtf(1 - s0);
  float q1 = (float)(n1 * 0.5 * m), q2 = (float)(n2 * 0.5 * m);
  // std::min(0.999999f, std::max(q, -0.999999f)): a NaN clamps to +0.999999.
  q1 = q1 < -0.999999f ? -0.999999f : q1;
  q1 = q1 < 0.999999f ? q1 : 0.999999f;
  q2 = q2 < -0.999999f ? -0.999999f : q2;
  q2 = q2 < 0.999999f ? q2 : 0.999999f;
  const uint32_t iq1 = (uint32_t)((q1 + 1) * 32767.f), iq2 = (uint32_t)((q2 + 1) * 32767.f);
  return (iq1 << 16) | iq2;
}

// The kernel's decode (kernel_functions.cu:3592-3601, decode_factor 32767) in
// an exact short form: for every 16-bit iq, (float)((double)iq * (1/32767))
// equals the IEEE quotient (float)iq / 32767.f, and 1 - 2s rounded once in
// float equals (float)(1.0 - 2.0 * s), the double difference being exact.
__device__ __forceinline__ void Decode(uint32_t code, float n[3]) {
  const double kInv = 1.0 / 32767.0;
  const float q1 = (float)((double)(code >> 16) * kInv) - 1.0f;
  const float q2 = (float)((double)(code & 0x0000ffffu) * kInv) - 1.0f;
  const float s = fmaf(q1, q1, q2 * q2);
  const float root = sqrtf(1 - s);
  n[0] = 1.0f - 2.0f * s;
  n[1] = 2 * q1 * root;
  n[2] = 2 * q2 * root;
}

// Forward projection into a source view (kernel_functions.cu:3630-3640).
__device__ __forceinline__ void Project(const float4* rec, const float X[3], float* scol, float* srow) {
  const float4 p0 = rec[0], p1 = rec[1], p2 = rec[2];  // P rows
  const float ifz = 1.0f / Affine3(p2.x, p2.y, p2.z, X, p2.w);
  *scol = ifz * Affine3(p0.x, p0.y, p0.z, X, p0.w);
  *srow = ifz * Affine3(p1.x, p1.y, p1.z, X, p1.w);
}

// Point sample at (x + 0.5, y + 0.5), border zero: texel floor(x + 0.5).
__device__ __forceinline__ bool Texel(float scol, float srow, int w, int h, int* q) {
  const float fx = floorf(scol + 0.5f), fy = floorf(srow + 0.5f);
  if (!(fx >= 0.0f && fx < (float)w && fy >= 0.0f && fy < (float)h)) return false;
  *q = (int)fy * w + (int)fx;
  return true;
}

// Back-projection into the reference view (kernel_functions.cu:3650-3673).
__device__ __forceinline__ float BackProject(const float4* rec, const float refK[4], float scol, float srow, float sd,
                                             int col, int row, float* err) {
  const float4 q0 = rec[3], q1 = rec[4], q2 = rec[5];  // P^-1 rows
  const float x[3] = {scol * sd, srow * sd, sd};
  const float bx = Affine3(q0.x, q0.y, q0.z, x, q0.w);
  const float by = Affine3(q1.x, q1.y, q1.z, x, q1.w);
  const float bz = Affine3(q2.x, q2.y, q2.z, x, q2.w);
  const float ibz = 1.0f / bz;
  const float bcol = ibz * fmaf(refK[0], bx, refK[1] * bz);
  const float brow = ibz * fmaf(refK[2], by, refK[3] * bz);
  const float dc = (float)col - bcol, dr = (float)row - brow;
  *err = sqrtf(fmaf(dc, dc, dr * dr));
  return bz;
}

// The reference compares float depths with double constants (depth < 1e-6,
// src_depth < 1e-4); for a float x, (double)x < 1e-6 is x <= 1e-6f and
// (double)x < 1e-4 is x <= 1e-4f (no float lies between each constant and
// its float rounding, which is below it), so the tests stay in float.
__device__ __forceinline__ bool BelowDepthEps(float x) { return x <= 1e-6f; }
__device__ __forceinline__ bool BelowSrcEps(float x) { return x <= 1e-4f; }

// BubbleSort (src/mvs/utils.h:205-221).
__device__ __forceinline__ void BubbleSort(float* v, int n) {
  for (int i = 0; i < n - 1; ++i)
    for (int j = 0; j < n - 1 - i; ++j) {
      const float a = v[j], b = v[j + 1];
      if (a > b) { v[j] = b; v[j + 1] = a; }
    }
}

__device__ __forceinline__ bool PixelOf(const CfJob& j, int local, int* col, int* row) {
  const int by = local / j.blocks_x, bx = local - by * j.blocks_x;
  *col = bx * kBlockX + (int)(threadIdx.x & (kBlockX - 1));
  *row = by * kBlockY + (int)(threadIdx.x / kBlockX);
  return *col < j.width && *row < j.height;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
// Planar 3*W*H normals -> codes.
__global__ void EncodeKernel(const float* __restrict__ n, size_t wh, uint32_t* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < wh; i += (size_t)gridDim.x * blockDim.x)
    out[i] = Encode(n[i], n[wh + i], n[2 * wh + i]);
}

__global__ void FillU32Kernel(uint32_t* __restrict__ p, size_t n, uint32_t v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

// CrossFilterKernel (kernel_functions.cu:3561-3778) for every problem at once.
__global__ void __launch_bounds__(kThreads) CrossFilterRunKernel(const CfJob* __restrict__ jobs,
                                                                 const int2* __restrict__ blocks, CfConsts c) {
  __shared__ CfJob sj;
  const int2 blk = __ldg(blocks + blockIdx.x);  // (problem, tile)
  StageJob(&sj, jobs + blk.x);
  __syncthreads();
  int col, row;
  if (!PixelOf(sj, blk.y, &col, &row)) return;
  const int W = sj.width, H = sj.height;
  const size_t pix = (size_t)row * W + col;
  const float depth = sj.depth[pix];
  if (BelowDepthEps(depth) || col < 3 || col > W - 3 || row < 3 || row > H - 3) { sj.out[pix] = 0.0f; return; }
  float rn[3];
  Decode(__ldg(sj.code + pix), rn);
  float vr[3] = {fmaf(sj.refiK[0], (float)col, sj.refiK[1]), fmaf(sj.refiK[2], (float)row, sj.refiK[3]), 1.0f};
  const float X[3] = {depth * vr[0], depth * vr[1], depth};
  const float nvr = sqrtf(Dot3(vr, vr));
  vr[0] /= nvr; vr[1] /= nvr; vr[2] /= nvr;
  if (Dot3(rn, vr) >= c.max_view_cos) { sj.out[pix] = 0.0f; return; }
  float depths[SMVS_CROSS_MAX_SRC + 1];
  int good = 0;
  depths[0] = depth;
  for (int i = 0; i < sj.num_src; ++i) {
    const float4* rec = reinterpret_cast<const float4*>(sj.rec[i]);
    const CfSrc& s = sj.src[i];
    float scol, srow;
    Project(rec, X, &scol, &srow);
    int q;
    if (!Texel(scol, srow, s.width, s.height, &q)) continue;  // border: depth 0 < 1e-4
    const float sd = __ldg(s.depth + q);
    if (BelowSrcEps(sd)) continue;
    float err;
    const float bz = BackProject(rec, sj.refK, scol, srow, sd, col, row, &err);
    const float dd = depth - bz;
    if (err > c.fmax_err || dd * dd > depth * depth * c.thr2) continue;
    float sn[3];
    Decode(__ldg(s.aux + q), sn);
    const float4 r0 = rec[6], r1 = rec[7], r2 = rec[8];  // R row-major, then padding
    // R^T n (kernel_functions.cu:3742-3747)
    const float Rc0[3] = {r0.x, r0.w, r1.z}, Rc1[3] = {r0.y, r1.x, r1.w}, Rc2[3] = {r0.z, r1.y, r2.x};
    const float rs[3] = {Dot3(Rc0, sn), Dot3(Rc1, sn), Dot3(Rc2, sn)};
    if (Dot3(rn, rs) < c.max_cos) continue;
    depths[++good] = bz;
  }
  const int nth = (int)(good * 0.5);
  if (good >= sj.min_cons) {
    BubbleSort(depths, good);  // [quirk] entries [0, good) of good + 1 (:3766)
    sj.out[pix] = depths[nth];
  } else {
    sj.out[pix] = 0.0f;
  }
}

// DeduplicFilterKernel (kernel_functions.cu:3780-3916) for the problems of one level.
__global__ void __launch_bounds__(kThreads) DedupKernel(const CfJob* __restrict__ jobs,
                                                        const int2* __restrict__ blocks, CfConsts c) {
  __shared__ CfJob sj;
  const int2 blk = __ldg(blocks + blockIdx.x);  // (problem, tile)
  StageJob(&sj, jobs + blk.x);
  __syncthreads();
  int col, row;
  if (!PixelOf(sj, blk.y, &col, &row)) return;
  const int W = sj.width, H = sj.height;
  const size_t pix = (size_t)row * W + col;
  const float depth = sj.depth[pix];
  if (BelowDepthEps(depth) || col < 3 || col > W - 3 || row < 3 || row > H - 3) { sj.vis[pix] = 0u; return; }
  const uint32_t vis0 = sj.vis[pix];
  if (!(vis0 >> 3)) { sj.vis[pix] = 0u; return; }  // [quirk] :3803 shifts by sizeof(uint32_t) - 1
  const float X[3] = {depth * fmaf(sj.refiK[0], (float)col, sj.refiK[1]),
                      depth * fmaf(sj.refiK[2], (float)row, sj.refiK[3]), depth};
  float dd[SMVS_CROSS_MAX_SRC];
  int good = 0, num_vis = 0;
  uint32_t bits = vis0;
  for (int i = 0; i < sj.num_src; ++i) {
    const float4* rec = reinterpret_cast<const float4*>(sj.rec[i]);
    const CfSrc& s = sj.src[i];
    float scol, srow;
    Project(rec, X, &scol, &srow);
    int q;
    if (!Texel(scol, srow, s.width, s.height, &q)) continue;  // border: depth 0
    const float sd = __ldg(s.depth + q);
    if (sd == 0.0f) continue;
    float err;
    const float bz = BackProject(rec, sj.refK, scol, srow, sd, col, row, &err);
    const float d = depth - bz;
    if (err > c.fmax_err || d * d > depth * depth * c.thr2) continue;
    dd[good++] = fabsf(bz - depth);
    bits |= 1u << (SMVS_CROSS_MAX_SRC - 1 - i);
    // Another problem's writes to this layer finished in an earlier launch.
    if ((s.aux[q] & kVisKeep) && s.ref_flag) ++num_vis;
  }
  if (good < sj.min_cons || num_vis > 0) { sj.vis[pix] = 0u; return; }
  sj.vis[pix] = bits;
  const int nth = (int)((good - 1) * 0.5);
  BubbleSort(dd, good - 1);  // [quirk] entries [0, good - 1) of good (:3913)
  sj.out[pix] = dd[nth] / (c.thr * depth);
}

// GetDeduplicDepthMapsLayer (kernel_functions.cu:3943-3960).
__global__ void DedupDepthKernel(const float* __restrict__ depth, const uint32_t* __restrict__ vis, size_t wh,
                                 float* __restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < wh; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (vis[i] & kVisKeep) ? depth[i] : 0.0f;
}

int GridFor(size_t n) {
  const size_t b = (n + 255) / 256;
  return (int)std::max<size_t>(1, std::min<size_t>(b, 148 * 16));
}

// Stream-ordered pool per device; freed blocks stay cached for the next filter
// (smvs_cross_filter_release_cache returns them).
cudaMemPool_t DevicePool(int device) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(device);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[device] = pool;
  return pool;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host object
// ---------------------------------------------------------------------------
struct smvs_cross_filter {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaMemPool_t pool = nullptr;
  smvs_options opt;
  std::vector<smvs_filter_view> views;  // host copy of the metadata (map pointers cleared)
  std::vector<std::vector<int>> srcs;   // per problem
  std::vector<int> refs;                // per problem
  std::vector<size_t> off;              // element offset of each view's region
  size_t total = 0;
  float* d_depth = nullptr;
  uint32_t* d_code = nullptr;
  float* d_refined = nullptr;
  float* d_delta = nullptr;
  uint32_t* d_vis = nullptr;
  float* d_scratch = nullptr;  // 3 x largest view: host normal staging, dedup depth maps
  CfJob* d_jobs = nullptr;
  int2* d_blocks = nullptr;
  size_t job_capacity = 0, block_capacity = 0;
  std::vector<uint8_t> has_normal;          // per view
  std::vector<uint8_t> refined, dedup_ref;  // per view
  bool deduped = false;
  int dedup_levels = 0;
  int64_t launches = 0;
  std::vector<CfJob> h_jobs;
  std::vector<int2> h_blocks;
  // Profiling: (kind, start, stop) per timed launch, harvested on demand.
  bool profiling = false;
  struct Timed { int kind; cudaEvent_t a, b; };
  std::vector<Timed> timed;
  int prof_count[3] = {0, 0, 0};
  double prof_ms[3] = {0, 0, 0};
};

namespace {

// Brackets one launch on the filter's stream with events when profiling.
struct ProfScope {
  smvs_cross_filter* f;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(smvs_cross_filter* f_, int kind_) : f(f_), kind(kind_) {
    if (!f->profiling) return;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) { a = b = nullptr; return; }
    cudaEventRecord(a, f->stream);
  }
  ~ProfScope() {
    if (!a) return;
    cudaEventRecord(b, f->stream);
    f->timed.push_back({kind, a, b});
  }
};

void Harvest(smvs_cross_filter* f) {
  for (auto& t : f->timed) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      f->prof_count[t.kind] += 1;
      f->prof_ms[t.kind] += ms;
    }
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  f->timed.clear();
}

template <typename T>
int PoolAlloc(smvs_cross_filter* f, T** p, size_t bytes) {
  cudaError_t err = cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), std::max<size_t>(bytes, 16), f->pool,
                                            f->stream);
  if (err != cudaSuccess) {
    *p = nullptr;
    return Fail(SMVS_ENOMEM, "cross filter: device allocation of %zu bytes: %s", bytes, cudaGetErrorString(err));
  }
  return SMVS_OK;
}

template <typename T>
void PoolFree(smvs_cross_filter* f, T*& p) {
  if (p) cudaFreeAsync(p, f->stream);
  p = nullptr;
}

void FreeAll(smvs_cross_filter* f) {
  Harvest(f);
  if (f->pool) {
    PoolFree(f, f->d_depth);
    PoolFree(f, f->d_code);
    PoolFree(f, f->d_refined);
    PoolFree(f, f->d_delta);
    PoolFree(f, f->d_vis);
    PoolFree(f, f->d_scratch);
    PoolFree(f, f->d_jobs);
    PoolFree(f, f->d_blocks);
  }
  if (f->own_stream && f->stream) {
    cudaStreamSynchronize(f->stream);
    cudaStreamDestroy(f->stream);
  }
}

CfConsts MakeConsts(const smvs_options& o) {
  CfConsts c;
  c.fmax_err = (float)o.filter_geom_consistency_max_cost;
  c.thr = o.depth_diff_threshold;
  c.thr2 = c.thr * c.thr;
  // DEG2RAD(x) = x * 0.0174532925199432 (kernel_functions.h:39), evaluated in
  // double and passed to cosf as float, as the kernel's expressions do.
  c.max_view_cos = cosf((float)(100 * 0.0174532925199432));
  c.max_cos = cosf((float)((double)(float)o.max_normal_error * 0.0174532925199432));
  return c;
}

// InitTransforms (:1320-1407) for one problem: the reference K, its inverse
// and the sources' P, P^-1 and R from the 43-float pose records (no source
// scaling in the cross filter).
void FillJob(const smvs_cross_filter* f, int p, CfJob* j) {
  memset(j, 0, sizeof(*j));
  const smvs_filter_view& rv = f->views[f->refs[p]];
  j->width = rv.width;
  j->height = rv.height;
  j->num_src = (int)f->srcs[p].size();
  j->min_cons = std::min(f->opt.filter_min_num_consistent, j->num_src);
  j->blocks_x = (rv.width + kBlockX - 1) / kBlockX;
  j->refK[0] = rv.K[0]; j->refK[1] = rv.K[2]; j->refK[2] = rv.K[4]; j->refK[3] = rv.K[5];
  j->refiK[0] = 1.0f / j->refK[0];
  j->refiK[1] = -j->refK[1] / j->refK[0];
  j->refiK[2] = 1.0f / j->refK[2];
  j->refiK[3] = -j->refK[3] / j->refK[2];
  smvs_view ref{}, src{};
  memcpy(ref.K, rv.K, sizeof(ref.K)); memcpy(ref.R, rv.R, sizeof(ref.R)); memcpy(ref.T, rv.T, sizeof(ref.T));
  ref.scale = 1.0f;
  for (int i = 0; i < j->num_src; ++i) {
    const smvs_filter_view& sv = f->views[f->srcs[p][i]];
    memcpy(src.K, sv.K, sizeof(src.K)); memcpy(src.R, sv.R, sizeof(src.R)); memcpy(src.T, sv.T, sizeof(src.T));
    src.scale = 1.0f;
    float pose[SMVS_POSE_FLOATS];
    smvs_internal_pose_record(&ref, &src, pose);
    memcpy(j->rec[i], pose + 19, 12 * sizeof(float));       // P
    memcpy(j->rec[i] + 12, pose + 31, 12 * sizeof(float));  // P^-1
    memcpy(j->rec[i] + 24, pose + 4, 9 * sizeof(float));    // R
    j->src[i].width = sv.width;
    j->src[i].height = sv.height;
    j->src[i].ref_flag = sv.ref_flag ? 1 : 0;
  }
}

int EnsureJobs(smvs_cross_filter* f, size_t jobs, size_t blocks) {
  if (jobs <= f->job_capacity && blocks <= f->block_capacity) return SMVS_OK;
  PoolFree(f, f->d_jobs);  // stream-ordered: earlier launches still read the old arrays
  PoolFree(f, f->d_blocks);
  f->job_capacity = f->block_capacity = 0;
  int st = PoolAlloc(f, &f->d_jobs, std::max<size_t>(jobs, 1) * sizeof(CfJob));
  if (!st) st = PoolAlloc(f, &f->d_blocks, std::max<size_t>(blocks, 1) * sizeof(int2));
  if (st) return st;
  f->job_capacity = jobs;
  f->block_capacity = blocks;
  return SMVS_OK;
}

// Uploads f->h_jobs once and launches `kernel` once per segment, segment k
// being jobs [bounds[k], bounds[k + 1]), in stream order. A segment's blocks
// are listed (problem, tile) in row-band-major order: band 0 of every problem,
// then band 1, and so on. The host arrays may be rebuilt as soon as this
// returns: copies from pageable memory are staged before cudaMemcpyAsync
// returns.
template <typename Kernel>
int LaunchSegments(smvs_cross_filter* f, const std::vector<size_t>& bounds, Kernel kernel, int kind,
                   const CfConsts& c) {
  const size_t nseg = bounds.size() - 1, njobs = f->h_jobs.size();
  f->h_blocks.clear();
  std::vector<size_t> seg_start(nseg + 1, 0);
  for (size_t k = 0; k < nseg; ++k) {
    seg_start[k] = f->h_blocks.size();
    int bands = 0;
    for (size_t i = bounds[k]; i < bounds[k + 1]; ++i)
      bands = std::max(bands, (f->h_jobs[i].height + kBlockY - 1) / kBlockY);
    for (int by = 0; by < bands; ++by)
      for (size_t i = bounds[k]; i < bounds[k + 1]; ++i) {
        const CfJob& j = f->h_jobs[i];
        if (by >= (j.height + kBlockY - 1) / kBlockY) continue;
        for (int bx = 0; bx < j.blocks_x; ++bx) f->h_blocks.push_back(make_int2((int)(i - bounds[k]), by * j.blocks_x + bx));
      }
    if (f->h_blocks.size() - seg_start[k] > 0x7fffffffu)
      return Fail(SMVS_EINVAL, "cross filter: too many pixel blocks in one launch");
  }
  seg_start[nseg] = f->h_blocks.size();
  if (njobs == 0) return SMVS_OK;
  int st = EnsureJobs(f, njobs, f->h_blocks.size());
  if (st) return st;
  CF_CUDA(cudaMemcpyAsync(f->d_jobs, f->h_jobs.data(), njobs * sizeof(CfJob), cudaMemcpyHostToDevice, f->stream));
  CF_CUDA(cudaMemcpyAsync(f->d_blocks, f->h_blocks.data(), f->h_blocks.size() * sizeof(int2), cudaMemcpyHostToDevice,
                          f->stream));
  (void)cudaGetLastError();
  for (size_t k = 0; k < nseg; ++k) {
    const size_t nb = seg_start[k + 1] - seg_start[k];
    if (nb == 0) continue;
    ProfScope prof(f, kind);
    kernel<<<(unsigned)nb, kThreads, 0, f->stream>>>(f->d_jobs + bounds[k], f->d_blocks + seg_start[k], c);
    CF_CUDA(cudaGetLastError());
    ++f->launches;
  }
  return SMVS_OK;
}

int CopyOut(smvs_cross_filter* f, const void* dsrc, void* out, size_t bytes) {
  CF_CUDA(cudaMemcpyAsync(out, dsrc, bytes, cudaMemcpyDefault, f->stream));
  CF_CUDA(cudaStreamSynchronize(f->stream));
  return SMVS_OK;
}

int CheckView(const smvs_cross_filter* f, int view) {
  if (!f) return Fail(SMVS_EINVAL, "null cross filter");
  if (view < 0 || view >= (int)f->views.size()) return Fail(SMVS_EINVAL, "view %d out of range", view);
  return SMVS_OK;
}

// The zero-filled refined buffer (allocated on first use).
int EnsureRefined(smvs_cross_filter* f) {
  if (f->d_refined) return SMVS_OK;
  int st = PoolAlloc(f, &f->d_refined, f->total * 4);
  if (st) return st;
  CF_CUDA(cudaMemsetAsync(f->d_refined, 0, f->total * 4, f->stream));
  return SMVS_OK;
}

}  // namespace

// The pool above, for the other units that allocate per call.
cudaMemPool_t smvs_internal_device_pool(int device) { return DevicePool(device); }

extern "C" {

int smvs_cross_filter_create(const smvs_options* opt, const smvs_filter_view* views, int num_views,
                             const smvs_filter_problem* problems, int num_problems, int memory, void* stream,
                             smvs_cross_filter** out) {
  if (!opt || !views || !out || num_views < 1 || num_problems < 0 || (num_problems > 0 && !problems))
    return Fail(SMVS_EINVAL, "cross filter: null argument or empty view set");
  *out = nullptr;
  if (memory != SMVS_MEM_HOST && memory != SMVS_MEM_DEVICE) return Fail(SMVS_EINVAL, "cross filter: bad memory kind");
  if (!(opt->filter_geom_consistency_max_cost >= 0) || !(opt->depth_diff_threshold >= 0))
    return Fail(SMVS_EINVAL, "cross filter: thresholds must be >= 0");
  if (opt->filter_min_num_consistent < 0) return Fail(SMVS_EINVAL, "filter_min_num_consistent must be >= 0");
  bool any_normal = false;
  for (int v = 0; v < num_views; ++v) {
    const smvs_filter_view& fv = views[v];
    // Pixel indices are 32-bit inside the kernels.
    if (fv.width < 1 || fv.height < 1 || (size_t)fv.width * fv.height >= ((size_t)1 << 31))
      return Fail(SMVS_EINVAL, "cross filter: view %d has bad size %dx%d", v, fv.width, fv.height);
    if (!fv.depth) return Fail(SMVS_EINVAL, "cross filter: view %d has no depth map", v);
    any_normal |= fv.normal != nullptr;
  }
  std::vector<int> ref_of(num_views, -1);
  for (int p = 0; p < num_problems; ++p) {
    const smvs_filter_problem& pr = problems[p];
    if (pr.ref < 0 || pr.ref >= num_views) return Fail(SMVS_EINVAL, "cross filter: problem %d reference out of range", p);
    if (pr.num_src < 0 || pr.num_src > SMVS_CROSS_MAX_SRC)
      return Fail(SMVS_EINVAL, "cross filter: problem %d has %d sources (max %d)", p, pr.num_src, SMVS_CROSS_MAX_SRC);
    if (pr.num_src > 0 && !pr.src) return Fail(SMVS_EINVAL, "cross filter: problem %d has no source list", p);
    for (int i = 0; i < pr.num_src; ++i)
      if (pr.src[i] < 0 || pr.src[i] >= num_views || pr.src[i] == pr.ref)
        return Fail(SMVS_EINVAL, "cross filter: problem %d source %d is invalid", p, i);
    if (ref_of[pr.ref] >= 0)
      return Fail(SMVS_EINVAL, "cross filter: problems %d and %d share reference view %d", ref_of[pr.ref], p, pr.ref);
    ref_of[pr.ref] = p;
  }
  auto* f = new smvs_cross_filter();
  f->opt = *opt;
  f->views.assign(views, views + num_views);
  f->has_normal.resize(num_views);
  for (int v = 0; v < num_views; ++v) f->has_normal[v] = views[v].normal != nullptr;
  for (int p = 0; p < num_problems; ++p) {
    f->refs.push_back(problems[p].ref);
    f->srcs.emplace_back(problems[p].src, problems[p].src + problems[p].num_src);
  }
  f->off.resize(num_views);
  size_t max_wh = 0;
  for (int v = 0; v < num_views; ++v) {
    f->off[v] = f->total;
    const size_t wh = (size_t)views[v].width * views[v].height;
    f->total += (wh + 31) & ~(size_t)31;  // 128-byte aligned regions
    max_wh = std::max(max_wh, wh);
  }
  f->refined.assign(num_views, 0);
  f->dedup_ref.assign(num_views, 0);
  auto fail = [&](int st) { FreeAll(f); delete f; return st; };
  if (opt->gpu_index >= 0) {
    cudaError_t err = cudaSetDevice(opt->gpu_index);
    if (err != cudaSuccess) return fail(Fail(SMVS_ECUDA, "cudaSetDevice(%d): %s", opt->gpu_index, cudaGetErrorString(err)));
  }
  cudaGetDevice(&f->device);
  if (stream) {
    f->stream = (cudaStream_t)stream;
  } else {
    cudaError_t err = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) return fail(Fail(SMVS_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(err)));
    f->own_stream = true;
  }
  f->pool = DevicePool(f->device);
  if (!f->pool) return fail(Fail(SMVS_ECUDA, "cross filter: no memory pool on device %d", f->device));
  int st;
  if ((st = PoolAlloc(f, &f->d_depth, f->total * 4))) return fail(st);
  if (any_normal && (st = PoolAlloc(f, &f->d_code, f->total * sizeof(uint32_t)))) return fail(st);
  if ((st = PoolAlloc(f, &f->d_scratch, max_wh * 3 * sizeof(float)))) return fail(st);
  // InitDepthMaps / InitNormalMaps (:1139-1258): one dense region per view.
  const cudaMemcpyKind kind = memory == SMVS_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  for (int v = 0; v < num_views; ++v) {
    const smvs_filter_view& fv = views[v];
    const size_t wh = (size_t)fv.width * fv.height;
    cudaError_t err = cudaMemcpyAsync(f->d_depth + f->off[v], fv.depth, wh * 4, kind, f->stream);
    if (err != cudaSuccess) return fail(Fail(SMVS_ECUDA, "cross filter: depth upload: %s", cudaGetErrorString(err)));
    if (fv.normal) {
      const float* n = fv.normal;
      if (memory == SMVS_MEM_HOST) {  // stage the planar map through the scratch buffer
        err = cudaMemcpyAsync(f->d_scratch, fv.normal, wh * 12, cudaMemcpyHostToDevice, f->stream);
        if (err != cudaSuccess) return fail(Fail(SMVS_ECUDA, "cross filter: normal upload: %s", cudaGetErrorString(err)));
        n = f->d_scratch;
      }
      (void)cudaGetLastError();
      EncodeKernel<<<GridFor(wh), 256, 0, f->stream>>>(n, wh, f->d_code + f->off[v]);
      err = cudaGetLastError();
      if (err != cudaSuccess) return fail(Fail(SMVS_ECUDA, "cross filter: normals: %s", cudaGetErrorString(err)));
      ++f->launches;
    }
    f->views[v].depth = nullptr;
    f->views[v].normal = nullptr;
  }
  if (memory == SMVS_MEM_HOST) {
    // Host maps may be pinned (copied asynchronously): they are free to reuse
    // once this call returns, as with the reference's synchronous upload.
    cudaError_t err = cudaStreamSynchronize(f->stream);
    if (err != cudaSuccess) return fail(Fail(SMVS_ECUDA, "cross filter: upload: %s", cudaGetErrorString(err)));
  }
  *out = f;
  return SMVS_OK;
}

int smvs_cross_filter_run(smvs_cross_filter* f) {
  if (!f) return Fail(SMVS_EINVAL, "null cross filter");
  cudaSetDevice(f->device);
  const int np = (int)f->refs.size();
  for (int p = 0; p < np; ++p) {
    if (f->srcs[p].empty()) continue;
    if (!f->has_normal[f->refs[p]]) return Fail(SMVS_EINVAL, "cross filter: view %d has no normal map", f->refs[p]);
    for (int s : f->srcs[p])
      if (!f->has_normal[s]) return Fail(SMVS_EINVAL, "cross filter: view %d has no normal map", s);
  }
  int st = EnsureRefined(f);
  if (st) return st;
  f->h_jobs.clear();
  for (int p = 0; p < np; ++p) {
    if (f->srcs[p].empty()) continue;  // :1504-1506
    CfJob j;
    FillJob(f, p, &j);
    const int r = f->refs[p];
    j.depth = f->d_depth + f->off[r];
    j.code = f->d_code + f->off[r];
    j.out = f->d_refined + f->off[r];
    for (int i = 0; i < j.num_src; ++i) {
      const int s = f->srcs[p][i];
      j.src[i].depth = f->d_depth + f->off[s];
      j.src[i].aux = f->d_code + f->off[s];
    }
    f->h_jobs.push_back(j);
  }
  st = LaunchSegments(f, {0, f->h_jobs.size()}, CrossFilterRunKernel, SMVS_CF_KERNEL_RUN, MakeConsts(f->opt));
  if (st) return st;
  for (int p = 0; p < np; ++p)
    if (!f->srcs[p].empty()) f->refined[f->refs[p]] = 1;
  return SMVS_OK;
}

int smvs_cross_filter_dedup_run(smvs_cross_filter* f) {
  if (!f) return Fail(SMVS_EINVAL, "null cross filter");
  if (f->opt.filter_min_num_consistent < 1)
    return Fail(SMVS_EINVAL, "dedup needs filter_min_num_consistent >= 1 (the reference reads an unset entry otherwise)");
  cudaSetDevice(f->device);
  const int nv = (int)f->views.size(), np = (int)f->refs.size();
  int st;
  if (!f->d_vis && (st = PoolAlloc(f, &f->d_vis, f->total * 4))) return st;
  if (!f->d_delta && (st = PoolAlloc(f, &f->d_delta, f->total * 4))) return st;
  bool any_flag = false;
  for (int v = 0; v < nv; ++v) any_flag |= f->views[v].ref_flag != 0;
  if (any_flag && (st = EnsureRefined(f))) return st;
  // ResetDepthMaps (:1260-1318): ref_flag views read their refined map; one
  // that no problem refined reads zeros (its region was zero-filled).
  auto input = [&](int v) -> const float* {
    return f->views[v].ref_flag ? f->d_refined + f->off[v] : f->d_depth + f->off[v];
  };
  (void)cudaGetLastError();
  {
    ProfScope prof(f, SMVS_CF_KERNEL_OTHER);
    FillU32Kernel<<<GridFor(f->total), 256, 0, f->stream>>>(f->d_vis, f->total, kVisKeep);  // FillGpuMat :3930-3941
  }
  CF_CUDA(cudaGetLastError());
  ++f->launches;
  CF_CUDA(cudaMemsetAsync(f->d_delta, 0, f->total * 4, f->stream));
  // Levels: a problem runs after every earlier problem that writes a layer it
  // reads or writes, or reads the layer it writes.
  std::vector<int> last_write(nv, 0), last_read(nv, 0), level(np, 0);
  int levels = 0;
  for (int p = 0; p < np; ++p) {
    if (f->srcs[p].empty()) continue;  // :1568-1570
    const int r = f->refs[p];
    int lv = std::max(last_write[r], last_read[r]);
    for (int s : f->srcs[p]) lv = std::max(lv, last_write[s]);
    level[p] = lv + 1;
    last_write[r] = level[p];
    for (int s : f->srcs[p]) last_read[s] = std::max(last_read[s], level[p]);
    levels = std::max(levels, level[p]);
  }
  f->h_jobs.clear();
  std::vector<size_t> bounds{0};
  for (int lv = 1; lv <= levels; ++lv) {
    for (int p = 0; p < np; ++p) {
      if (level[p] != lv) continue;
      CfJob j;
      FillJob(f, p, &j);
      const int r = f->refs[p];
      j.depth = input(r);
      j.vis = f->d_vis + f->off[r];
      j.out = f->d_delta + f->off[r];
      for (int i = 0; i < j.num_src; ++i) {
        const int s = f->srcs[p][i];
        j.src[i].depth = input(s);
        j.src[i].aux = f->d_vis + f->off[s];
      }
      f->h_jobs.push_back(j);
    }
    bounds.push_back(f->h_jobs.size());
  }
  // One launch per level on one stream: level lv sees every write of level lv - 1.
  st = LaunchSegments(f, bounds, DedupKernel, SMVS_CF_KERNEL_DEDUP, MakeConsts(f->opt));
  if (st) return st;
  std::fill(f->dedup_ref.begin(), f->dedup_ref.end(), 0);
  for (int p = 0; p < np; ++p)
    if (!f->srcs[p].empty()) f->dedup_ref[f->refs[p]] = 1;
  f->dedup_levels = levels;
  f->deduped = true;
  return SMVS_OK;
}

int smvs_cross_filter_get_refined_depth_map(smvs_cross_filter* f, int view, float* out) {
  int st = CheckView(f, view);
  if (st) return st;
  if (!out) return Fail(SMVS_EINVAL, "null output");
  if (!f->refined[view]) return Fail(SMVS_ESTATE, "view %d was not refined by smvs_cross_filter_run", view);
  cudaSetDevice(f->device);
  return CopyOut(f, f->d_refined + f->off[view], out, (size_t)f->views[view].width * f->views[view].height * 4);
}

int smvs_cross_filter_get_dedup_depth_map(smvs_cross_filter* f, int view, float* out) {
  int st = CheckView(f, view);
  if (st) return st;
  if (!out) return Fail(SMVS_EINVAL, "null output");
  if (!f->deduped) return Fail(SMVS_ESTATE, "smvs_cross_filter_dedup_run has not run");
  cudaSetDevice(f->device);
  const size_t wh = (size_t)f->views[view].width * f->views[view].height;
  const float* in = f->views[view].ref_flag ? f->d_refined + f->off[view] : f->d_depth + f->off[view];
  (void)cudaGetLastError();
  {
    ProfScope prof(f, SMVS_CF_KERNEL_OTHER);
    DedupDepthKernel<<<GridFor(wh), 256, 0, f->stream>>>(in, f->d_vis + f->off[view], wh, f->d_scratch);
  }
  CF_CUDA(cudaGetLastError());
  ++f->launches;
  return CopyOut(f, f->d_scratch, out, wh * 4);
}

int smvs_cross_filter_get_delta_depth_map(smvs_cross_filter* f, int view, float* out) {
  int st = CheckView(f, view);
  if (st) return st;
  if (!out) return Fail(SMVS_EINVAL, "null output");
  if (!f->deduped || !f->dedup_ref[view]) return Fail(SMVS_ESTATE, "view %d was not a dedup reference", view);
  cudaSetDevice(f->device);
  return CopyOut(f, f->d_delta + f->off[view], out, (size_t)f->views[view].width * f->views[view].height * 4);
}

int smvs_cross_filter_get_visibility_map(smvs_cross_filter* f, int view, uint32_t* out) {
  int st = CheckView(f, view);
  if (st) return st;
  if (!out) return Fail(SMVS_EINVAL, "null output");
  if (!f->deduped) return Fail(SMVS_ESTATE, "smvs_cross_filter_dedup_run has not run");
  cudaSetDevice(f->device);
  return CopyOut(f, f->d_vis + f->off[view], out, (size_t)f->views[view].width * f->views[view].height * 4);
}

int smvs_cross_filter_get_device_maps(smvs_cross_filter* f, int view, const float** refined, const float** delta,
                                      const uint32_t** visibility) {
  int st = CheckView(f, view);
  if (st) return st;
  if (refined) *refined = f->refined[view] ? f->d_refined + f->off[view] : nullptr;
  if (delta) *delta = (f->deduped && f->dedup_ref[view]) ? f->d_delta + f->off[view] : nullptr;
  if (visibility) *visibility = f->deduped ? f->d_vis + f->off[view] : nullptr;
  return SMVS_OK;
}

int smvs_cross_filter_set_profiling(smvs_cross_filter* f, int enable) {
  if (!f) return Fail(SMVS_EINVAL, "null cross filter");
  f->profiling = enable != 0;
  return SMVS_OK;
}

int smvs_cross_filter_get_profile(smvs_cross_filter* f, int kind, int* count, double* total_ms) {
  if (!f || kind < 0 || kind > 2) return Fail(SMVS_EINVAL, "bad cross filter profile query");
  cudaSetDevice(f->device);
  Harvest(f);
  if (count) *count = f->prof_count[kind];
  if (total_ms) *total_ms = f->prof_ms[kind];
  return SMVS_OK;
}

int64_t smvs_cross_filter_launch_count(smvs_cross_filter* f) { return f ? f->launches : -1; }

int smvs_cross_filter_dedup_levels(smvs_cross_filter* f) { return f ? f->dedup_levels : -1; }

int smvs_cross_filter_synchronize(smvs_cross_filter* f) {
  if (!f) return Fail(SMVS_EINVAL, "null cross filter");
  cudaSetDevice(f->device);
  CF_CUDA(cudaStreamSynchronize(f->stream));
  return SMVS_OK;
}

void smvs_cross_filter_destroy(smvs_cross_filter* f) {
  if (!f) return;
  cudaSetDevice(f->device);
  FreeAll(f);
  delete f;
}

int smvs_cross_filter_release_cache(int gpu_index) {
  int dev = gpu_index;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return Fail(SMVS_ECUDA, "no current device");
  cudaMemPool_t pool = DevicePool(dev);
  if (!pool) return Fail(SMVS_ECUDA, "no memory pool on device %d", dev);
  CF_CUDA(cudaDeviceSynchronize());
  CF_CUDA(cudaMemPoolTrimTo(pool, 0));
  return SMVS_OK;
}

}  // extern "C"
