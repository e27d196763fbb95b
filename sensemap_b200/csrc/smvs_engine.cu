// smvs_engine.cu — host engine behind the C ABI (include/smvs.h).
//
// One smvs_engine replaces one sensemap::mvs::PatchMatchACMMCuda instance
// (src/mvs/patch_match_cuda.h:154-203). Differences in structure, not in
// results: per-engine parameter block instead of __constant__ slots, one
// stream with no host synchronisation between kernels (the reference syncs
// after every launch, src/util/cudacc.cc:50-64), per-view pitched textures
// instead of one layered cudaArray, and status codes instead of exit().
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/smvs.h"
#include "../../include/smvs_testing.h"
#include "smvs_device.cuh"
#include "smvs_kernels.h"

cudaMemPool_t smvs_internal_device_pool(int device);

namespace {

thread_local std::string g_last_error;

int Fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define SMVS_CUDA(call)                                                                       \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return Fail(SMVS_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

size_t StorageBytes(int storage) {
  return storage == SMVS_STORE_U8 ? 1 : (storage == SMVS_STORE_F16 ? 2 : 4);
}

// Host pose algebra of InitTransforms (patch_match_cuda.cu:493-580) with
// ComputeRelativePose / ComputeProjectionCenter / ComposeProjectionMatrix /
// ComposeInverseProjectionMatrix (src/mvs/utils.cc:14-52), composed in FP64
// and rounded to the 43-float record once.
void BuildPoseRecord(const smvs_view& ref, const smvs_view& s, float* o) {
  double iK[9];
  for (int k = 0; k < 9; ++k) iK[k] = s.K[k];
  const double scale = (s.scale > 0.f) ? s.scale : 1.0;
  if (scale != 1.0) { iK[0] *= scale; iK[2] *= scale; iK[4] *= scale; iK[5] *= scale; }
  double R[9], T[3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += (double)s.R[r * 3 + k] * (double)ref.R[c * 3 + k];
      R[r * 3 + c] = acc;  // R2 * R1^T
    }
  for (int r = 0; r < 3; ++r)
    T[r] = (double)s.T[r] - (R[r * 3] * ref.T[0] + R[r * 3 + 1] * ref.T[1] + R[r * 3 + 2] * ref.T[2]);
  double C[3];
  for (int r = 0; r < 3; ++r) C[r] = -(R[r] * T[0] + R[3 + r] * T[1] + R[6 + r] * T[2]);
  double P[12];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += iK[r * 3 + k] * (c < 3 ? R[k * 3 + c] : T[k]);
      P[r * 4 + c] = acc;
    }
  // [P; 0 0 0 1]^-1 = [R^T K^-1 | -R^T T] for an upper-triangular pinhole K.
  double Ki[9] = {0};
  Ki[0] = 1.0 / iK[0];
  Ki[1] = -iK[1] / (iK[0] * iK[4]);
  Ki[2] = (iK[1] * iK[5] - iK[2] * iK[4]) / (iK[0] * iK[4]);
  Ki[4] = 1.0 / iK[4];
  Ki[5] = -iK[5] / iK[4];
  Ki[8] = 1.0;
  double iP[12];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) {
      double acc = 0;
      for (int k = 0; k < 3; ++k) acc += R[k * 3 + r] * Ki[k * 3 + c];
      iP[r * 4 + c] = acc;
    }
    iP[r * 4 + 3] = -(R[r] * T[0] + R[3 + r] * T[1] + R[6 + r] * T[2]);
  }
  o[0] = (float)iK[0]; o[1] = (float)iK[2]; o[2] = (float)iK[4]; o[3] = (float)iK[5];
  for (int k = 0; k < 9; ++k) o[4 + k] = (float)R[k];
  for (int k = 0; k < 3; ++k) o[13 + k] = (float)T[k];
  for (int k = 0; k < 3; ++k) o[16 + k] = (float)C[k];
  for (int k = 0; k < 12; ++k) o[19 + k] = (float)P[k];
  for (int k = 0; k < 12; ++k) o[31 + k] = (float)iP[k];
}

cudaError_t MakeTexture(void* ptr, int storage_or_float, int w, int h, size_t pitch, cudaTextureObject_t* tex) {
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = ptr;
  rd.res.pitch2D.width = (size_t)w;
  rd.res.pitch2D.height = (size_t)h;
  rd.res.pitch2D.pitchInBytes = pitch;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeBorder;
  td.addressMode[1] = cudaAddressModeBorder;
  td.addressMode[2] = cudaAddressModeBorder;
  td.filterMode = cudaFilterModeLinear;
  td.normalizedCoords = 0;
  if (storage_or_float == SMVS_STORE_U8) {
    rd.res.pitch2D.desc = cudaCreateChannelDesc<uint8_t>();
    td.readMode = cudaReadModeNormalizedFloat;
  } else if (storage_or_float == SMVS_STORE_F16) {
    rd.res.pitch2D.desc = cudaCreateChannelDescHalf();
    td.readMode = cudaReadModeElementType;
  } else {
    rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
    td.readMode = cudaReadModeElementType;
  }
  return cudaCreateTextureObject(tex, &rd, &td, nullptr);
}

}  // namespace

struct smvs_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  smvs_options opt;
  int W = 0, H = 0, N = 0;
  bool ran = false;
  bool filtered = false;
  int64_t launches = 0;
  smvs::JobParams jp;
  std::vector<void*> allocations;
  std::vector<cudaTextureObject_t> textures;
  float* d_ref = nullptr;
  float* d_ref_sum = nullptr;
  float* d_ref_sqsum = nullptr;
  float* d_grad = nullptr;
  float* d_poses = nullptr;
  float* d_depth = nullptr;
  float* d_normal = nullptr;
  float* d_conf = nullptr;
  float* d_cost = nullptr;
  uint32_t* d_view_sel = nullptr;
  float* d_init_depth = nullptr;   // ref.depth as given (init / RunFilter input)
  float* d_init_normal = nullptr;  // ref.normal as given
  uint8_t* d_mask = nullptr;
  uint16_t* d_curv = nullptr;   // 2*W*H (est_curvature && geom_consistency)
  float* d_prior_wgt = nullptr;   // ref_prior_wgt as given (has_prior_depth)
  float* d_prior = nullptr;       // W*H projected prior depth (propagate_depth)
  float* d_composite = nullptr;   // N*W*H projected depths per source (propagate_depth)
  std::vector<int> src_w, src_h;  // source sizes (the propagate-depth projection grid)
  std::vector<const float*> src_depth;  // pitched device copies of the sources' depth maps (NULL = none)
  std::vector<size_t> src_depth_pitch;
  // One-job batch for the checkerboard kernels: [JobParams | iters | prefix | conf prefix].
  void* d_batch = nullptr;
  CUtensorMap* d_tmap = nullptr;  // the reference image's TMA descriptor
  int* d_status = nullptr;        // bounded waits of the kernels that gave up
  bool use_tma = true;
  int persistent = 0;             // thread-per-pixel kernels as a persistent grid (smvs_tuning)
  bool tma_active = false;        // the last run staged reference tiles with TMA
  int tpp_used = 0;               // threads per pixel of the last run
  int tma_polls = 0;              // TMA tile wait bound (0 = default; a test hook shortens it)
  int tma_skip_copy = 0;          // test hook: issue no tile copy, so the waits run out
  float* d_ggrad = nullptr;     // W*H (median_filter)
  bool has_init = false;
  bool has_src_depth = false;
  // Optional per-launch timing (smvs_set_profiling): CUDA events around each
  // kernel, grouped by kind (smvs_kernel_kind).
  bool profiling = false;
  struct Timed { int kind; cudaEvent_t start, stop; };
  std::vector<Timed> timed;

  // Memory the library's per-device memory pool keeps in reserve (freed by
  // pools, filters and fusion) is returned to the device before an allocation
  // here reports that the device is full.
  static bool ReleaseReserve() {
    (void)cudaGetLastError();
    int dev = 0;
    cudaMemPool_t pool = cudaGetDevice(&dev) == cudaSuccess ? smvs_internal_device_pool(dev) : nullptr;
    return pool && cudaDeviceSynchronize() == cudaSuccess && cudaMemPoolTrimTo(pool, 0) == cudaSuccess;
  }
  int Alloc(void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation && ReleaseReserve()) e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return Fail(SMVS_ENOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    allocations.push_back(*p);
    return SMVS_OK;
  }
  int AllocPitch(void** p, size_t* pitch, size_t wbytes, int h) {
    cudaError_t e = cudaMallocPitch(p, pitch, wbytes, (size_t)h);
    if (e == cudaErrorMemoryAllocation && ReleaseReserve()) e = cudaMallocPitch(p, pitch, wbytes, (size_t)h);
    if (e != cudaSuccess) return Fail(SMVS_ENOMEM, "cudaMallocPitch failed: %s", cudaGetErrorString(e));
    allocations.push_back(*p);
    return SMVS_OK;
  }
  ~smvs_engine() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& t : timed) { cudaEventDestroy(t.start); cudaEventDestroy(t.stop); }
    for (auto t : textures) cudaDestroyTextureObject(t);
    for (auto p : allocations) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

// Upload `bytes` of a host or device buffer to a fresh device buffer.
int StageIn(smvs_engine* e, const void* src, size_t bytes, int memory, void** dst) {
  if (memory == SMVS_MEM_DEVICE) {
    *dst = const_cast<void*>(src);
    return SMVS_OK;
  }
  int st = e->Alloc(dst, bytes);
  if (st) return st;
  SMVS_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, e->stream));
  return SMVS_OK;
}

size_t ViewStride(const smvs_view& v) {
  if (v.row_stride) return v.row_stride;
  return (size_t)v.width * (v.pixel_format == SMVS_PIX_U8 ? 1 : 4);
}

int CheckLaunch(smvs_engine* e, cudaError_t err, const char* what) {
  if (err != cudaSuccess) return Fail(SMVS_ECUDA, "%s launch failed: %s", what, cudaGetErrorString(err));
  e->launches++;
  return SMVS_OK;
}

// Launch `fn` (returning cudaError_t) as kernel kind `kind`, bracketed by
// events when profiling is on.
template <typename Fn>
int Launch(smvs_engine* e, int kind, const char* what, Fn fn) {
  // Clear a launch error another library may have left on this thread, so a
  // failure is only reported against the launch that caused it.
  (void)cudaGetLastError();
  cudaEvent_t a = nullptr, b = nullptr;
  if (e->profiling) {
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
      return Fail(SMVS_ECUDA, "cudaEventCreate failed");
    cudaEventRecord(a, e->stream);
  }
  int st = CheckLaunch(e, fn(), what);
  if (e->profiling) {
    cudaEventRecord(b, e->stream);
    e->timed.push_back({kind, a, b});
  }
  return st;
}

int CheckView(const smvs_view& v, const char* what) {
  if (v.width <= 0 || v.height <= 0 || !v.pixels)
    return Fail(SMVS_EINVAL, "%s: empty image (width=%d height=%d)", what, v.width, v.height);
  if (v.pixel_format != SMVS_PIX_U8 && v.pixel_format != SMVS_PIX_F32)
    return Fail(SMVS_EINVAL, "%s: unknown pixel format %d", what, v.pixel_format);
  if (v.K[0] == 0.f || v.K[4] == 0.f) return Fail(SMVS_EINVAL, "%s: zero focal length", what);
  return SMVS_OK;
}

}  // namespace

// Fill the iteration-dependent and tiling fields of a job's parameters.
int smvs_internal_prepare_job(smvs::JobParams* p, const smvs_options* o) {
  p->seed = o->random_seed;
  p->num_iterations = o->num_iterations;
  p->local_opt = o->local_optimization && !o->has_prior_depth;
  for (int it = 0; it < smvs::kMaxIterations; ++it)  // patch_match_cuda.cu:778-779
    p->th_tab[it] = (float)o->init_ncc_matching_cost * expf(-(float)(it * it) / (float)o->alpha);
  p->blocks_x = (p->W + 2 * p->block_x - 1) / (2 * p->block_x);
  p->conf_blocks_x = (p->W + 31) / 32;
  // Threads per pixel: the requested value, raised until the block's cost
  // matrices fit in shared memory (maps do not depend on it).
  // Jobs with a prior run the thread-per-pixel kernels, which alone carry the
  // prior paths.
  const int want = p->prior_mode != 0 ? 1 : (p->tpp > 0 ? p->tpp : 1);
  const int tpp = smvs::FitThreadsPerPixel(p->R, smvs::ViewBucket(p->N), p->block_x, want);
  if (!tpp)
    return Fail(SMVS_EINVAL, "no launch shape with sweep_block_x=%d fits %d source views in shared memory",
                p->block_x, p->N);
  p->tpp = tpp;
  return SMVS_OK;
}

// The 43-float pose record of one source view, for the other entry points of
// this library.
void smvs_internal_pose_record(const smvs_view* ref, const smvs_view* src, float* out43) {
  BuildPoseRecord(*ref, *src, out43);
}

extern "C" {

const char* smvs_last_error(void) { return g_last_error.c_str(); }

// Lets the host-only I/O unit report through the same thread-local slot.
void smvs_internal_set_error(const char* msg) { g_last_error = msg ? msg : ""; }

int smvs_options_default(smvs_options* o) {
  if (!o) return Fail(SMVS_EINVAL, "null options");
  memset(o, 0, sizeof(*o));
  o->depth_min = -1.0;
  o->depth_max = -1.0;
  o->window_radius = 5;
  o->window_step = 2;
  o->sigma_spatial = 5.0;  // = window_radius at struct init (patch_match_options.h:89)
  o->sigma_color = 0.2f;
  o->num_samples = 15;
  o->num_iterations = 5;
  o->geom_consistency = 1;
  o->geom_consistency_regularizer = 0.3f;
  o->geom_consistency_max_cost = 3.0f;
  o->filter = 1;
  o->filter_min_num_consistent = 1;
  o->filter_geom_consistency_max_cost = 1.0f;
  o->max_normal_error = 15.0f;
  o->init_depth_random = 0;  // = !geom_consistency (patch_match_options.h:164)
  o->random_depth_ratio = 0.004f;
  o->random_angle1_range = (float)(20.0 * M_PI / 180.0);
  o->random_angle2_range = (float)(12.0 * M_PI / 180.0);
  o->init_ncc_matching_cost = 0.8f;
  o->max_ncc_matching_cost = 1.2f;
  o->alpha = 90.0f;
  o->beta = 0.3f;
  o->thk = 4;
  o->num_good_hypothesis = 2;
  o->num_bad_hypothesis = 3;
  o->random_optimization = 1;
  o->local_optimization = 1;
  o->est_curvature = 0;
  o->median_filter = 0;
  o->conf_filter = 0;
  o->depth_diff_threshold = 0.02f;
  o->conf_threshold = 0.5f;
  o->has_prior_depth = 0;
  o->propagate_depth = 0;
  o->random_seed = 0;
  o->image_storage = SMVS_STORE_U8;
  o->gpu_index = -1;
  return SMVS_OK;
}

int smvs_options_check(const smvs_options* o) {
  if (!o) return Fail(SMVS_EINVAL, "null options");
  // PatchMatchOptions::Check (patch_match_options.cc:75-101).
  if (o->depth_min > o->depth_max && !(o->depth_min == -1.0 && o->depth_max == -1.0))
    return Fail(SMVS_EINVAL, "depth_min > depth_max");
  if (o->depth_min < 0 || o->depth_max <= 0) return Fail(SMVS_EINVAL, "depth range must be set (depth_min >= 0, depth_max > 0)");
  if (o->window_radius <= 0 || o->window_radius > 32) return Fail(SMVS_EINVAL, "window_radius out of range");
  if (o->window_step <= 0 || o->window_step > 2) return Fail(SMVS_EINVAL, "window_step out of range");
  if (!(o->sigma_spatial > 0) || !(o->sigma_color > 0)) return Fail(SMVS_EINVAL, "sigmas must be > 0");
  if (o->num_samples <= 0) return Fail(SMVS_EINVAL, "num_samples must be > 0");
  if (o->num_iterations < 0) return Fail(SMVS_EINVAL, "num_iterations must be >= 0");
  if (o->geom_consistency_regularizer < 0 || o->geom_consistency_max_cost < 0)
    return Fail(SMVS_EINVAL, "geometric consistency weights must be >= 0");
  if (o->filter_min_num_consistent < 0) return Fail(SMVS_EINVAL, "filter_min_num_consistent must be >= 0");
  // Engine limits. The reference silently computes (5,2) windows for any
  // other pair (kernel_functions.cu:1394-1399) while its reference moments use
  // the requested pair; this engine rejects such pairs instead.
  if (!smvs::SupportedWindow(o->window_radius, o->window_step))
    return Fail(SMVS_EINVAL, "window (radius=%d, step=%d) not supported: use (3|5|7,1) or (3|4|5|7,2)",
                o->window_radius, o->window_step);
  if (o->thk < 1 || o->thk > 4) return Fail(SMVS_EINVAL, "thk must be in 1..4 (mweights, kernel_functions.cu:22)");
  // patch_match_cuda.cu:946-947: the two prior paths share one set of buffers.
  if (o->has_prior_depth && o->propagate_depth)
    return Fail(SMVS_EINVAL, "has_prior_depth and propagate_depth exclude each other");
  // The propagate-depth initialisation lives in the given-map branch of
  // InitWorkspace (patch_match_cuda.cu:593-603), and its projections read the
  // source depth maps that the geometric pass would use
  // (patch_match_cuda.cu:318-377); the controller never combines them
  // (patch_match_controller.cc:3611-3613).
  if (o->propagate_depth && o->init_depth_random)
    return Fail(SMVS_EINVAL, "propagate_depth needs init_depth_random == 0");
  if (o->propagate_depth && o->geom_consistency)
    return Fail(SMVS_EINVAL, "propagate_depth excludes geom_consistency");
  if (o->num_iterations > smvs::kMaxIterations)
    return Fail(SMVS_EINVAL, "num_iterations must be <= %d", smvs::kMaxIterations);
  if (o->image_storage < SMVS_STORE_U8 || o->image_storage > SMVS_STORE_F32)
    return Fail(SMVS_EINVAL, "unknown image_storage %d", o->image_storage);
  return SMVS_OK;
}

int smvs_create(const smvs_options* opt, const smvs_problem* prob, void* stream, smvs_engine** out) {
  if (!out) return Fail(SMVS_EINVAL, "null output handle");
  *out = nullptr;
  int st = smvs_options_check(opt);
  if (st) return st;
  if (!prob) return Fail(SMVS_EINVAL, "null problem");
  if (prob->num_src < 1 || prob->num_src > SMVS_MAX_SRC)
    return Fail(SMVS_EINVAL, "num_src=%d outside 1..%d", prob->num_src, SMVS_MAX_SRC);
  if (!prob->src) return Fail(SMVS_EINVAL, "null source view list");
  if ((st = CheckView(prob->ref, "reference view"))) return st;
  for (int i = 0; i < prob->num_src; ++i)
    if ((st = CheckView(prob->src[i], "source view"))) return st;
  if (opt->geom_consistency)
    for (int i = 0; i < prob->num_src; ++i)
      if (!prob->src[i].depth) return Fail(SMVS_EINVAL, "geom_consistency needs every source view's depth map");
  if (opt->has_prior_depth && (!prob->ref.depth || !prob->ref.normal))
    return Fail(SMVS_EINVAL, "has_prior_depth needs the reference view's depth and normal maps (ref.depth, ref.normal)");
  if (!opt->init_depth_random && (!prob->ref.depth || !prob->ref.normal) && opt->num_iterations >= 0) {
    // Run() with init_depth_random == 0 starts from the given maps
    // (patch_match_cuda.cu:593-601); RunFilter needs ref.depth only.
  }

  auto* e = new smvs_engine();
  e->opt = *opt;
  if (opt->gpu_index >= 0) {
    cudaError_t err = cudaSetDevice(opt->gpu_index);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "cudaSetDevice(%d): %s", opt->gpu_index, cudaGetErrorString(err)); }
  }
  cudaGetDevice(&e->device);
  {
    const cudaError_t err = smvs::ConfigureKernels();
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "kernel set-up: %s", cudaGetErrorString(err)); }
  }
  if (stream) {
    e->stream = (cudaStream_t)stream;
  } else {
    cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(err)); }
    e->own_stream = true;
  }
  const int W = prob->ref.width, H = prob->ref.height, N = prob->num_src;
  e->W = W; e->H = H; e->N = N;
  const size_t WH = (size_t)W * H;
  smvs::JobParams& p = e->jp;
  memset(&p, 0, sizeof(p));
  p.W = W; p.H = H; p.N = N; p.R = opt->window_radius; p.S = opt->window_step;
  const float ss = (float)opt->sigma_spatial, sc = (float)opt->sigma_color;
  p.sn = 1.0f / (2.0f * ss * ss);
  p.cn = 1.0f / (2.0f * sc * sc);
  p.depth_min = (float)opt->depth_min;
  p.depth_max = (float)opt->depth_max;
  p.rand_depth_ratio = opt->random_depth_ratio;
  p.rand_a1 = opt->random_angle1_range;
  p.rand_a2 = opt->random_angle2_range;
  p.max_mc = (float)opt->max_ncc_matching_cost;
  const float beta = (float)opt->beta;
  p.inv_beta2 = 0.5f / (beta * beta);
  p.num_samples = opt->num_samples;
  p.num_good = opt->num_good_hypothesis;
  p.num_bad = opt->num_bad_hypothesis;
  p.random_opt = opt->random_optimization;
  p.geom = opt->geom_consistency;
  p.thk = opt->thk < N ? opt->thk : N;  // patch_match_cuda.cu:949-950
  p.block_x = 32;
  p.tpp = 1;
  p.geom_reg = (float)opt->geom_consistency_regularizer;
  p.geom_max = (float)opt->geom_consistency_max_cost;
  const float* K = prob->ref.K;
  p.refK[0] = K[0]; p.refK[1] = K[2]; p.refK[2] = K[4]; p.refK[3] = K[5];
  p.refiK[0] = 1.0f / p.refK[0];
  p.refiK[1] = -p.refK[1] / p.refK[0];
  p.refiK[2] = 1.0f / p.refK[2];
  p.refiK[3] = -p.refK[3] / p.refK[2];

#define TRY(x) do { int s_ = (x); if (s_) { delete e; return s_; } } while (0)
  // Pose records (InitTransforms).
  std::vector<float> poses((size_t)N * SMVS_POSE_FLOATS);
  for (int i = 0; i < N; ++i) BuildPoseRecord(prob->ref, prob->src[i], poses.data() + (size_t)i * SMVS_POSE_FLOATS);
  TRY(e->Alloc((void**)&e->d_poses, poses.size() * sizeof(float)));
  {
    cudaError_t err = cudaMemcpyAsync(e->d_poses, poses.data(), poses.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "pose upload: %s", cudaGetErrorString(err)); }
    // The host vector dies at return: make the copy complete first.
    err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "pose upload: %s", cudaGetErrorString(err)); }
  }
  p.poses = e->d_poses;

  // Reference image: uint8-quantised, normalised (patch_match_cuda.cu:110-147).
  TRY(e->Alloc((void**)&e->d_ref, WH * sizeof(float)));
  {
    void* staged = nullptr;
    const size_t stride = ViewStride(prob->ref);
    TRY(StageIn(e, prob->ref.pixels, stride * H, prob->memory, &staged));
    TRY(Launch(e, SMVS_KERNEL_CONVERT, "convert ref", [&] {
      return smvs::LaunchConvertImage(staged, prob->ref.pixel_format, stride, W, H, e->d_ref, 3, W * sizeof(float), 1,
                                      e->stream);
    }));
  }
  p.ref = e->d_ref;
  TRY(e->Alloc((void**)&e->d_ref_sum, WH * sizeof(float)));
  TRY(e->Alloc((void**)&e->d_ref_sqsum, WH * sizeof(float)));
  TRY(e->Alloc((void**)&e->d_grad, WH * sizeof(float)));
  p.ref_sum = e->d_ref_sum; p.ref_sqsum = e->d_ref_sqsum; p.grad = e->d_grad;
  TRY(Launch(e, SMVS_KERNEL_PREP, "prep ref",
             [&] { return smvs::LaunchPrepRef(p, e->d_ref_sum, e->d_ref_sqsum, e->d_grad, e->stream); }));

  // Source views (InitSourceImages, patch_match_cuda.cu:199-418).
  for (int i = 0; i < N; ++i) {
    const smvs_view& v = prob->src[i];
    void* dimg = nullptr;
    size_t pitch = 0;
    TRY(e->AllocPitch(&dimg, &pitch, (size_t)v.width * StorageBytes(opt->image_storage), v.height));
    void* staged = nullptr;
    const size_t stride = ViewStride(v);
    TRY(StageIn(e, v.pixels, stride * v.height, prob->memory, &staged));
    TRY(Launch(e, SMVS_KERNEL_CONVERT, "convert source", [&] {
      return smvs::LaunchConvertImage(staged, v.pixel_format, stride, v.width, v.height, dimg, opt->image_storage,
                                      pitch, 1, e->stream);
    }));
    cudaTextureObject_t tex = 0;
    cudaError_t err = MakeTexture(dimg, opt->image_storage, v.width, v.height, pitch, &tex);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "source texture: %s", cudaGetErrorString(err)); }
    e->textures.push_back(tex);
    p.src_tex[i] = tex;
    e->src_w.push_back(v.width);
    e->src_h.push_back(v.height);
    e->src_depth.push_back(nullptr);
    e->src_depth_pitch.push_back(0);
    if (v.depth) {
      float* dd = nullptr;
      size_t dpitch = 0;
      TRY(e->AllocPitch((void**)&dd, &dpitch, (size_t)v.width * sizeof(float), v.height));
      err = cudaMemcpy2DAsync(dd, dpitch, v.depth, (size_t)v.width * sizeof(float), (size_t)v.width * sizeof(float),
                              v.height, prob->memory == SMVS_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                              e->stream);
      if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "source depth upload: %s", cudaGetErrorString(err)); }
      err = MakeTexture(dd, SMVS_STORE_F32, v.width, v.height, dpitch, &tex);
      if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "depth texture: %s", cudaGetErrorString(err)); }
      e->textures.push_back(tex);
      p.dep_tex[i] = tex;
      e->src_depth.back() = dd;
      e->src_depth_pitch.back() = dpitch;
    }
  }
  e->has_src_depth = true;
  for (int i = 0; i < N; ++i) e->has_src_depth = e->has_src_depth && prob->src[i].depth != nullptr;

  // State maps.
  TRY(e->Alloc((void**)&e->d_depth, WH * sizeof(float)));
  TRY(e->Alloc((void**)&e->d_normal, 3 * WH * sizeof(float)));
  TRY(e->Alloc((void**)&e->d_conf, WH * sizeof(float)));
  TRY(e->Alloc((void**)&e->d_cost, (size_t)N * WH * sizeof(float)));
  TRY(e->Alloc((void**)&e->d_view_sel, WH * sizeof(uint32_t)));
  p.depth = e->d_depth; p.normal = e->d_normal; p.conf = e->d_conf; p.cost = e->d_cost; p.view_sel = e->d_view_sel;
  if (prob->ref.depth) {
    TRY(StageIn(e, prob->ref.depth, WH * sizeof(float), prob->memory, (void**)&e->d_init_depth));
    if (prob->ref.normal) TRY(StageIn(e, prob->ref.normal, 3 * WH * sizeof(float), prob->memory, (void**)&e->d_init_normal));
    e->has_init = (prob->ref.normal != nullptr);
  }
  if (prob->ref_mask) TRY(StageIn(e, prob->ref_mask, WH, prob->memory, (void**)&e->d_mask));
  // Prior maps (InitPriorDepthAndNormalInfo, patch_match_cuda.cu:715-746): the
  // reference view's given depth and normal maps and its optional weights.
  if (opt->has_prior_depth) {
    p.prior_mode = 1;
    p.prior_depth = e->d_init_depth;
    p.prior_normal = e->d_init_normal;
    if (prob->ref_prior_wgt) {
      TRY(StageIn(e, prob->ref_prior_wgt, WH * sizeof(float), prob->memory, (void**)&e->d_prior_wgt));
      p.prior_wgt = e->d_prior_wgt;
    }
  } else if (opt->propagate_depth) {
    // The reference's sweep reads prior normal and weight maps that this mode
    // never fills (0 x 0 buffers, patch_match_cuda.cu:588-591): here they read as 0.
    TRY(e->Alloc((void**)&e->d_prior, WH * sizeof(float)));
    TRY(e->Alloc((void**)&e->d_composite, (size_t)N * WH * sizeof(float)));
    p.prior_mode = 2;
    p.prior_depth = e->d_prior;
  }
  if (opt->est_curvature && opt->geom_consistency) TRY(e->Alloc((void**)&e->d_curv, 2 * WH * sizeof(uint16_t)));
  TRY(e->Alloc(&e->d_batch, sizeof(smvs::JobParams) + 8 * sizeof(int)));
  TRY(e->Alloc((void**)&e->d_tmap, sizeof(CUtensorMap)));
  TRY(e->Alloc((void**)&e->d_status, sizeof(int)));
  {
    cudaError_t err = cudaMemsetAsync(e->d_status, 0, sizeof(int), e->stream);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "status: %s", cudaGetErrorString(err)); }
  }
  if (opt->median_filter) TRY(e->Alloc((void**)&e->d_ggrad, WH * sizeof(float)));
  // Source pixels/depths staged from host memory must stay valid until the
  // copies complete; the caller's buffers are only guaranteed during this call.
  if (prob->memory == SMVS_MEM_HOST) {
    cudaError_t err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) { delete e; return Fail(SMVS_ECUDA, "upload: %s", cudaGetErrorString(err)); }
  }
#undef TRY
  *out = e;
  return SMVS_OK;
}

// The reference image's TMA descriptor for the job's launch shape, or
// tma_box_w = 0 (plain loads) when the image does not qualify.
static int UploadRefMap(smvs_engine* e, smvs::JobParams* p) {
  p->tma_box_w = p->tma_box_h = 0;
  CUtensorMap map;
  if (!e->use_tma || !smvs::EncodeRefMap(&map, p->ref, p->W, p->H, p->block_x, p->tpp, p->R)) return SMVS_OK;
  // The host descriptor dies at return: copy it before returning.
  SMVS_CUDA(cudaMemcpyAsync(e->d_tmap, &map, sizeof(map), cudaMemcpyHostToDevice, e->stream));
  SMVS_CUDA(cudaStreamSynchronize(e->stream));
  p->tma_box_w = smvs::RefTileW(p->block_x, p->R);
  p->tma_box_h = smvs::RefTileH(p->block_x, p->tpp, p->R);
  return SMVS_OK;
}

// Reports a kernel wait that gave up (the stream has been synchronised).
static int CheckStatus(smvs_engine* e) {
  int status = 0;
  SMVS_CUDA(cudaMemcpy(&status, e->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (status) return Fail(SMVS_ETIMEDOUT, "a reference-tile copy did not complete; maps of this run are incomplete");
  return SMVS_OK;
}

int smvs_run(smvs_engine* e) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  smvs::JobParams p = e->jp;
  const smvs_options& o = e->opt;
  const size_t WH = (size_t)e->W * e->H;
  cudaSetDevice(e->device);
  if (!o.init_depth_random) {
    if (!e->has_init) return Fail(SMVS_EINVAL, "init_depth_random == 0 needs ref.depth and ref.normal");
    SMVS_CUDA(cudaMemcpyAsync(e->d_depth, e->d_init_depth, WH * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
    SMVS_CUDA(cudaMemcpyAsync(e->d_normal, e->d_init_normal, 3 * WH * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
  }
  if (o.propagate_depth) {  // patch_match_cuda.cu:603-659
    int st = Launch(e, SMVS_KERNEL_INIT, "propagate-depth init", [&] {
      return smvs::LaunchPropagateInit(p, e->src_w.data(), e->src_h.data(),
                                       e->src_depth.data(), e->src_depth_pitch.data(), e->d_composite,
                                       e->d_prior, e->stream);
    });
    if (st) return st;
  }
  p.stage_key = smvs::StageKey(o.random_seed, smvs::kStageInit);
  int st = Launch(e, SMVS_KERNEL_INIT, "init", [&] {
    return smvs::LaunchInit(p, o.init_depth_random, (float)o.depth_min, (float)o.depth_max, e->stream);
  });
  if (st) return st;
  smvs::Batch b{};
  if ((st = smvs_internal_prepare_job(&p, &o))) return st;
  if ((st = UploadRefMap(e, &p))) return st;
  e->tma_active = p.tma_box_w > 0;
  e->tpp_used = p.tpp;
  {
    // The checkerboard kernels run as a batch of one job.
    char host[sizeof(smvs::JobParams) + 8 * sizeof(int)];
    int* ints = reinterpret_cast<int*>(host + sizeof(smvs::JobParams));
    memcpy(host, &p, sizeof(p));
    const int by = smvs::SweepRows(p.block_x, p.tpp);
    const int nb = p.blocks_x * ((e->H + by - 1) / by);
    const int ncb = p.conf_blocks_x * ((e->H + 7) / 8);
    ints[0] = 0;             // iteration counter
    ints[1] = 0; ints[2] = nb;   // checkerboard prefix
    ints[3] = 0; ints[4] = ncb;  // InitConf prefix
    SMVS_CUDA(cudaMemcpyAsync(e->d_batch, host, sizeof(host), cudaMemcpyHostToDevice, e->stream));
    char* dev = static_cast<char*>(e->d_batch);
    int* dints = reinterpret_cast<int*>(dev + sizeof(smvs::JobParams));
    b.jobs = reinterpret_cast<const smvs::JobParams*>(dev);
    b.iters = dints;
    b.block_start = dints + 1;
    b.conf_block_start = dints + 3;
    b.num_jobs = 1;
    b.total_blocks = nb;
    b.total_conf_blocks = ncb;
    b.block_x = p.block_x;
    b.tpp = p.tpp;
    b.R = p.R; b.S = p.S; b.NB = smvs::ViewBucket(p.N);
    b.ref_maps = e->d_tmap;
    b.status = e->d_status;
    b.tma_polls = e->tma_polls;
    b.tma_skip_copy = e->tma_skip_copy;
    b.persistent = e->persistent;
    b.grid_cap = smvs::PersistentGridCap();
  }
  if ((st = Launch(e, SMVS_KERNEL_INIT_CONF, "init conf", [&] { return smvs::LaunchInitConf(b, e->stream); }))) return st;
  int* iters = const_cast<int*>(b.iters);
  for (int iter = 0; iter < o.num_iterations; ++iter) {
    for (int colour = 0; colour < 2; ++colour)
      if ((st = Launch(e, SMVS_KERNEL_SWEEP, "sweep", [&] { return smvs::LaunchSweep(b, colour, e->stream); }))) return st;
    if (p.local_opt && iter > 2) {  // :861-880
      for (int colour = 0; colour < 2; ++colour)
        if ((st = Launch(e, SMVS_KERNEL_LOCAL_OPT, "local optimisation",
                         [&] { return smvs::LaunchLocalOpt(b, colour, e->stream); })))
          return st;
    }
    if ((st = Launch(e, SMVS_KERNEL_INIT, "advance", [&] { return smvs::LaunchAdvance(iters, 1, e->stream); }))) return st;
  }
  // Post-processing in the reference's order (patch_match_cuda.cu:985-1052).
  if (e->d_curv && (st = Launch(e, SMVS_KERNEL_POST, "curvature",
                                [&] { return smvs::LaunchCurvature(p, e->d_curv, e->stream); })))
    return st;
  if (o.median_filter) {
    if ((st = Launch(e, SMVS_KERNEL_POST, "geometric gradient",
                     [&] { return smvs::LaunchGeomGradient(p, e->d_ggrad, e->stream); })))
      return st;
    for (int colour = 0; colour < 2; ++colour)
      if ((st = Launch(e, SMVS_KERNEL_POST, "median filter", [&] {
             return smvs::LaunchMedianFilter(p, e->d_ggrad, o.depth_diff_threshold, colour, e->stream);
           })))
        return st;
  }
  if (o.filter && o.conf_filter)
    for (int colour = 0; colour < 2; ++colour)
      if ((st = Launch(e, SMVS_KERNEL_POST, "confidence filter", [&] {
             return smvs::LaunchConfFilter(p, o.depth_diff_threshold, o.conf_threshold, colour, e->stream);
           })))
        return st;
  if (e->d_mask && (st = Launch(e, SMVS_KERNEL_MASK, "mask", [&] { return smvs::LaunchMask(p, e->d_mask, e->stream); })))
    return st;
  e->ran = true;
  return SMVS_OK;
}

// Test hook: the propagate-depth initial maps alone (the given maps composited
// with the projected source depths, before random hypotheses fill the rest).
int smvs_test_propagate_init(smvs_engine* e, float* depth, float* normal, float* prior) {
  if (!e || !depth || !normal || !prior) return Fail(SMVS_EINVAL, "null argument");
  if (!e->opt.propagate_depth) return Fail(SMVS_EINVAL, "the engine was not created with propagate_depth");
  cudaSetDevice(e->device);
  const size_t WH = (size_t)e->W * e->H;
  const smvs::JobParams& p = e->jp;
  SMVS_CUDA(cudaMemcpyAsync(e->d_depth, e->d_init_depth, WH * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
  SMVS_CUDA(cudaMemcpyAsync(e->d_normal, e->d_init_normal, 3 * WH * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
  int st = Launch(e, SMVS_KERNEL_INIT, "propagate-depth init", [&] {
    return smvs::LaunchPropagateInit(p, e->src_w.data(), e->src_h.data(), e->src_depth.data(),
                                     e->src_depth_pitch.data(), e->d_composite, e->d_prior, e->stream);
  });
  if (st) return st;
  SMVS_CUDA(cudaMemcpyAsync(depth, e->d_depth, WH * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
  SMVS_CUDA(cudaMemcpyAsync(normal, e->d_normal, 3 * WH * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
  SMVS_CUDA(cudaMemcpyAsync(prior, e->d_prior, WH * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
  SMVS_CUDA(cudaStreamSynchronize(e->stream));
  return SMVS_OK;
}

int smvs_run_filter(smvs_engine* e, int dedup) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  if (!e->d_init_depth) return Fail(SMVS_EINVAL, "RunFilter needs the reference view's depth map (ref.depth)");
  if (!e->has_src_depth) return Fail(SMVS_EINVAL, "RunFilter needs every source view's depth map");
  cudaSetDevice(e->device);
  smvs::JobParams p = e->jp;
  const int min_cons = e->opt.filter_min_num_consistent < e->N ? e->opt.filter_min_num_consistent : e->N;
  int st = Launch(e, SMVS_KERNEL_FILTER, "filter depth maps", [&] {
    return smvs::LaunchFilterDepthMaps(p, e->d_init_depth, e->d_depth, min_cons,
                                       (float)e->opt.filter_geom_consistency_max_cost, dedup, e->stream);
  });
  if (st) return st;
  e->filtered = true;
  return SMVS_OK;
}

static int CopyOut(smvs_engine* e, void* dst, const void* src, size_t bytes, bool need_run) {
  if (!e || !dst) return Fail(SMVS_EINVAL, "null argument");
  if (need_run && !e->ran) return Fail(SMVS_ESTATE, "call smvs_run first");
  if (!need_run && !e->ran && !e->filtered) return Fail(SMVS_ESTATE, "call smvs_run or smvs_run_filter first");
  SMVS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, e->stream));
  SMVS_CUDA(cudaStreamSynchronize(e->stream));
  return CheckStatus(e);
}

int smvs_get_depth_map(smvs_engine* e, float* out) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  return CopyOut(e, out, e->d_depth, (size_t)e->W * e->H * sizeof(float), false);
}
int smvs_get_normal_map(smvs_engine* e, float* out) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  return CopyOut(e, out, e->d_normal, 3 * (size_t)e->W * e->H * sizeof(float), true);
}
int smvs_get_conf_map(smvs_engine* e, float* out) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  return CopyOut(e, out, e->d_conf, (size_t)e->W * e->H * sizeof(float), true);
}
int smvs_get_cost_map(smvs_engine* e, float* out) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  return CopyOut(e, out, e->d_cost, (size_t)e->N * e->W * e->H * sizeof(float), true);
}
int smvs_get_view_sel_map(smvs_engine* e, uint32_t* out) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  return CopyOut(e, out, e->d_view_sel, (size_t)e->W * e->H * sizeof(uint32_t), true);
}
int smvs_get_curvature_map(smvs_engine* e, uint16_t* out) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  if (!e->d_curv) return Fail(SMVS_EINVAL, "curvature map needs est_curvature and geom_consistency");
  return CopyOut(e, out, e->d_curv, 2 * (size_t)e->W * e->H * sizeof(uint16_t), true);
}
int smvs_get_size(const smvs_engine* e, int* w, int* h, int* n) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  if (w) *w = e->W;
  if (h) *h = e->H;
  if (n) *n = e->N;
  return SMVS_OK;
}
int smvs_get_device_maps(const smvs_engine* e, smvs_device_maps* m) {
  if (!e || !m) return Fail(SMVS_EINVAL, "null argument");
  m->width = e->W; m->height = e->H; m->num_src = e->N;
  m->depth = e->d_depth; m->normal = e->d_normal; m->conf = e->d_conf; m->cost = e->d_cost; m->view_sel = e->d_view_sel;
  return SMVS_OK;
}
int smvs_synchronize(smvs_engine* e) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  SMVS_CUDA(cudaStreamSynchronize(e->stream));
  return CheckStatus(e);
}
int64_t smvs_launch_count(const smvs_engine* e) { return e ? e->launches : -1; }

int smvs_set_tuning(smvs_engine* e, const smvs_tuning* t) {
  if (!e || !t) return Fail(SMVS_EINVAL, "null argument");
  const int bx = t->sweep_block_x;
  if (bx != 8 && bx != 16 && bx != 32 && bx != 64) return Fail(SMVS_EINVAL, "sweep_block_x must be 8, 16, 32 or 64");
  const int tpp = t->threads_per_pixel;
  if (tpp != 1 && tpp != 2 && tpp != 4) return Fail(SMVS_EINVAL, "threads_per_pixel must be 1, 2 or 4");
  if (!smvs::ValidSweepShape(bx, tpp)) return Fail(SMVS_EINVAL, "sweep_block_x * threads_per_pixel must be <= 256");
  e->jp.block_x = bx;
  e->jp.tpp = tpp;
  e->use_tma = t->ref_tile_tma != 0;
  e->persistent = t->persistent != 0;
  return SMVS_OK;
}

int smvs_get_tuning(const smvs_engine* e, smvs_tuning* t) {
  if (!e || !t) return Fail(SMVS_EINVAL, "null argument");
  t->sweep_block_x = e->jp.block_x;
  t->ref_tile_tma = e->tma_active ? 1 : 0;
  t->threads_per_pixel = e->tpp_used > 0 ? e->tpp_used : e->jp.tpp;
  t->persistent = t->threads_per_pixel == 1 ? e->persistent : 0;  // only the thread-per-pixel kernels loop
  return SMVS_OK;
}

int smvs_set_profiling(smvs_engine* e, int enable) {
  if (!e) return Fail(SMVS_EINVAL, "null engine");
  e->profiling = enable != 0;
  return SMVS_OK;
}

int smvs_get_profile(smvs_engine* e, int kind, int* count, double* total_ms) {
  if (!e || !count || !total_ms) return Fail(SMVS_EINVAL, "null argument");
  SMVS_CUDA(cudaStreamSynchronize(e->stream));
  int n = 0;
  double ms = 0;
  for (auto& t : e->timed) {
    if (t.kind != kind) continue;
    float x = 0.f;
    SMVS_CUDA(cudaEventElapsedTime(&x, t.start, t.stop));
    ms += x;
    ++n;
  }
  *count = n;
  *total_ms = ms;
  return SMVS_OK;
}
void smvs_destroy(smvs_engine* e) { delete e; }

int smvs_test_persistent_grid(int max_blocks) {
  if (max_blocks < 0) return Fail(SMVS_EINVAL, "persistent grid: bad arguments");
  smvs::SetPersistentGridCap(max_blocks);
  return SMVS_OK;
}

int smvs_test_tile_waits(smvs_engine* e, int polls, int skip_copy) {
  if (!e || polls < 0) return Fail(SMVS_EINVAL, "tile waits: bad arguments");
  e->tma_polls = polls;
  e->tma_skip_copy = skip_copy ? 1 : 0;
  return SMVS_OK;
}

// Launch-shape autotuner: times the checkerboard sweep of one iteration of
// `prob` for every candidate launch shape (pixels per block row x threads per
// pixel, and for one thread per pixel one block per tile or a persistent grid;
// reference tiles by TMA where the image qualifies) on a scratch engine, best
// of `repeats`, and returns the fastest. Results do not depend on the launch
// shape, so the choice only affects speed.
int smvs_autotune(const smvs_options* opt, const smvs_problem* prob, void* stream, int repeats, smvs_tuning* best,
                  smvs_tuning* tried, double* ms, int capacity, int* num_tried) {
  if (!opt || !prob || !best) return Fail(SMVS_EINVAL, "null argument");
  smvs_options o = *opt;
  o.num_iterations = 1;  // init, InitConf and both colours of one sweep
  smvs_engine* e = nullptr;
  int st = smvs_create(&o, prob, stream, &e);
  if (st) return st;
  const int xs[4] = {8, 16, 32, 64};
  const int ts[3] = {1, 2, 4};
  double best_ms = 0;
  int n = 0;
  std::vector<smvs_tuning> seen;
  for (int k = 0; k < 4 && st == SMVS_OK; ++k)
    for (int j = 0; j < 3 * 2 && st == SMVS_OK; ++j) {
      const int tpp = ts[j / 2], pers = j % 2;
      if (!smvs::ValidSweepShape(xs[k], tpp) || (pers && tpp != 1)) continue;
      smvs_tuning t{xs[k], 1, tpp, pers};
      if ((st = smvs_set_tuning(e, &t))) break;
      double t_best = 0;
      for (int r = 0; r < (repeats > 0 ? repeats : 3) && st == SMVS_OK; ++r) {
        if ((st = smvs_synchronize(e))) break;
        for (auto& ev : e->timed) { cudaEventDestroy(ev.start); cudaEventDestroy(ev.stop); }
        e->timed.clear();
        if ((st = smvs_set_profiling(e, 1)) || (st = smvs_run(e))) break;
        int cnt = 0;
        double tot = 0;
        if ((st = smvs_get_profile(e, SMVS_KERNEL_SWEEP, &cnt, &tot))) break;
        if (cnt > 0 && (r == 0 || tot / cnt < t_best)) t_best = tot / cnt;
      }
      if (st) break;
      smvs_tuning used;
      smvs_get_tuning(e, &used);
      bool dup = false;  // threads_per_pixel raised to fit: the same shape as an earlier candidate
      for (const auto& u : seen)
        dup = dup || (u.sweep_block_x == used.sweep_block_x && u.threads_per_pixel == used.threads_per_pixel &&
                      u.persistent == used.persistent);
      if (dup) continue;
      seen.push_back(used);
      if (tried && ms && n < capacity) {
        tried[n] = used;
        ms[n] = t_best;
      }
      ++n;
      if (n == 1 || t_best < best_ms) {
        best_ms = t_best;
        *best = used;
      }
    }
  if (num_tried) *num_tried = n;
  smvs_destroy(e);
  return st;
}

}  // extern "C"
