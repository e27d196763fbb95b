// ref_driver.cu — drives the REFERENCE's own PatchMatch kernels (compiled from
// the SenseMap sources by oracle/ref_build.py) on caller-supplied inputs.
//
// TEST INFRASTRUCTURE ONLY: the second oracle. It calls the reference's
// kernels (src/mvs/kernel_functions.cu, gpu_mat_ref_image.cu, gpu_mat_prng.cu)
// in the order PatchMatchACMMCuda::Run issues them (patch_match_cuda.cu:748-1057)
// with textures configured as InitRefImage / InitSourceImages / InitTransforms /
// Preprocess configure them (patch_match_cuda.cu:110-580, 448-491). The host
// pose records are supplied by the caller (the 43-float layout of :516-559).
#include <cfloat>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "mvs/cuda_array_wrapper.h"
#include "mvs/gpu_mat_prng.h"
#include "mvs/gpu_mat_ref_image.h"
#include "mvs/kernel_functions.h"
#undef MAX_NUM_SRC_IMAGE
#define MAX_NUM_SRC_IMAGE 32  // as compiled by ref_kernels_n32.cu

using namespace sensemap;
using namespace sensemap::mvs;

extern "C" {

struct RefJob {
  int W, H, N;
  const uint8_t* ref;
  const uint8_t* const* src;
  const int* src_w;
  const int* src_h;
  const float* poses;
  float refK[4], refiK[4];
  int R, S;
  float sigma_s, sigma_c;
  float depth_min, depth_max;
  int num_iterations, geom, init_depth_random, local_opt, random_opt, num_samples, thk, good, bad;
  float geom_reg, geom_max, rand_depth_ratio, a1, a2, init_mc, max_mc, alpha, beta;
  const float* init_depth;
  const float* init_normal;
  const float* const* src_depth;  // per source; an entry may be NULL (propagate_depth: no map)
  int prior_mode;                 // 0 none, 1 has_prior_depth, 2 propagate_depth
  const float* prior_wgt;         // W*H or NULL (has_prior_depth)
};

struct RefOut {
  float* depth;
  float* normal;
  float* conf;
  float* cost;
  uint32_t* view_sel;
};

int ref_max_num_src(void) { return MAX_NUM_SRC_IMAGE; }

}  // extern "C"

namespace {

cudaTextureObject_t MakeArrayTexture(cudaArray* arr, cudaTextureFilterMode filter, cudaTextureReadMode read) {
  cudaResourceDesc resDesc;
  memset(&resDesc, 0, sizeof(resDesc));
  resDesc.resType = cudaResourceTypeArray;
  resDesc.res.array.array = arr;
  cudaTextureDesc texDesc;
  memset(&texDesc, 0, sizeof(texDesc));
  texDesc.addressMode[0] = cudaAddressModeBorder;
  texDesc.addressMode[1] = cudaAddressModeBorder;
  texDesc.addressMode[2] = cudaAddressModeBorder;
  texDesc.filterMode = filter;
  texDesc.readMode = read;
  texDesc.normalizedCoords = 0;
  cudaTextureObject_t t = 0;
  CUDA_SAFE_CALL(cudaCreateTextureObject(&t, &resDesc, &texDesc, NULL));
  return t;
}

struct Textures {
  std::unique_ptr<GpuMatRefImage> ref_image;
  std::unique_ptr<CudaArrayWrapper<uint8_t>> ref_dev, src_dev;
  std::unique_ptr<CudaArrayWrapper<float>> src_depth_dev, poses_dev, sum_dev, sqsum_dev;
  cudaTextureObject_t ref_tex = 0, src_tex = 0, src_depth_tex = 0, poses_tex = 0, sum_tex = 0, sqsum_tex = 0;
  ~Textures() {
    for (auto t : {ref_tex, src_tex, src_depth_tex, poses_tex, sum_tex, sqsum_tex})
      if (t) cudaDestroyTextureObject(t);
  }
};

void SetupTextures(const RefJob& j, Textures& t, bool with_images) {
  if (with_images) {
    // InitRefImage, patch_match_cuda.cu:110-147.
    t.ref_image.reset(new GpuMatRefImage(j.W, j.H));
    t.ref_image->Filter(j.ref, j.R, j.S, j.sigma_s, j.sigma_c);
    t.ref_dev.reset(new CudaArrayWrapper<uint8_t>(j.W, j.H, 1));
    t.ref_dev->CopyFromGpuMat(*t.ref_image->image);
    t.ref_tex = MakeArrayTexture(t.ref_dev->GetPtr(), cudaFilterModePoint, cudaReadModeNormalizedFloat);
  }
  size_t max_w = 0, max_h = 0;
  for (int i = 0; i < j.N; ++i) {
    max_w = std::max<size_t>(max_w, j.src_w[i]);
    max_h = std::max<size_t>(max_h, j.src_h[i]);
  }
  if (with_images) {
    // InitSourceImages, patch_match_cuda.cu:229-278.
    std::vector<uint8_t> packed(max_w * max_h * j.N, 0);
    for (int i = 0; i < j.N; ++i)
      for (int r = 0; r < j.src_h[i]; ++r)
        memcpy(packed.data() + max_w * max_h * i + r * max_w, j.src[i] + (size_t)r * j.src_w[i], j.src_w[i]);
    t.src_dev.reset(new CudaArrayWrapper<uint8_t>(max_w, max_h, j.N));
    t.src_dev->CopyToDevice(packed.data());
    t.src_tex = MakeArrayTexture(t.src_dev->GetPtr(), cudaFilterModeLinear, cudaReadModeNormalizedFloat);
  }
  if (j.src_depth) {
    // InitSourceImages geometric branch, patch_match_cuda.cu:318-367, and the
    // propagate-depth branch :377-417 (a source without a map stays 0).
    std::vector<float> packed(max_w * max_h * j.N, 0.f);
    for (int i = 0; i < j.N; ++i)
      for (int r = 0; j.src_depth[i] && r < j.src_h[i]; ++r)
        memcpy(packed.data() + max_w * max_h * i + r * max_w, j.src_depth[i] + (size_t)r * j.src_w[i],
               sizeof(float) * j.src_w[i]);
    t.src_depth_dev.reset(new CudaArrayWrapper<float>(max_w, max_h, j.N));
    t.src_depth_dev->CopyToDevice(packed.data());
    t.src_depth_tex = MakeArrayTexture(t.src_depth_dev->GetPtr(), cudaFilterModeLinear, cudaReadModeElementType);
  }
  // InitTransforms, patch_match_cuda.cu:503-579.
  SetRefK(j.refK, 0);
  SetRefInvK(j.refiK, 0);
  t.poses_dev.reset(new CudaArrayWrapper<float>(K_NUM_TFORM_PARAMS, j.N, 1));
  t.poses_dev->CopyToDevice(j.poses);
  t.poses_tex = MakeArrayTexture(t.poses_dev->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);
}

// Every pitched row cleared (the reference's GpuMat::FillWithScalar is a byte
// cudaMemset of width * height * depth * sizeof(T) bytes from the start of a
// pitched allocation, gpu_mat.h:240-243, which leaves the last rows of a map
// whose pitch exceeds its row size uninitialised).
void ClearMap(GpuMat<float>& m) {
  CUDA_SAFE_CALL(cudaMemset2D(m.GetPtr(), m.GetPitch(), 0, m.GetWidth() * sizeof(float), m.GetHeight() * m.GetDepth()));
}

// The propagate-depth initial maps in the reference's order
// (patch_match_cuda.cu:603-659): GenerateProjectDepthMaps per source with a
// map, CompositeInitDepthMap, CompositeInitNormalMap. The reference launches
// them with 32x32 blocks; the driver uses 32x16 (every kernel indexes pixels
// from blockDim and the projections combine by atomicMin, so results do not
// depend on the block shape) and checks every launch.
// The reference starts the projections from composite_depth_map.FillWithScalar
// (FLT_MAX), a byte cudaMemset of the float converted to int (gpu_mat.h:240-243):
// its fill byte is 0xff (every float NaN, which the atomicMin and the
// (0, FLT_MAX) test treat like FLT_MAX) when the host compiler folds the
// conversion, and 0x00 (no projection is ever stored, the mode does nothing)
// when it converts at run time. The driver fills FLT_MAX itself: the intended
// result.
int PropagateInit(const RefJob& j, const Textures& t, GpuMatPRNG& rand_state, GpuMat<float>& depth_map,
                  GpuMat<float>& normal_map, GpuMat<float>& prior_depth) {
  size_t max_w = 0, max_h = 0;
  for (int i = 0; i < j.N; ++i) {
    max_w = std::max<size_t>(max_w, j.src_w[i]);
    max_h = std::max<size_t>(max_h, j.src_h[i]);
  }
  const dim3 b(THREADS_PER_BLOCK, THREADS_PER_BLOCK / 2);
  GpuMat<float> composite(j.W, j.H, j.N);
  {
    std::vector<float> init((size_t)j.W * j.H * j.N, FLT_MAX);
    composite.CopyToDevice(init.data(), j.W * sizeof(float));
  }
  for (int i = 0; i < j.N; ++i) {
    if (!j.src_depth || !j.src_depth[i]) continue;
    const dim3 g((max_w - 1) / b.x + 1, (max_h - 1) / b.y + 1);
    GenerateProjectDepthMaps<<<g, b>>>(max_w, max_h, i, j.N, composite, t.src_depth_tex, t.poses_tex, 0);
    if (cudaGetLastError() != cudaSuccess) return 20;
  }
  CUDA_SYNC_AND_CHECK();
  // The reference clears its prior map with FillWithScalar(0)
  // (patch_match_cuda.cu:644-645); the driver clears all of it.
  ClearMap(prior_depth);
  const dim3 g((j.W - 1) / b.x + 1, (j.H - 1) / b.y + 1);
  CompositeInitDepthMap<<<g, b>>>(rand_state, depth_map, prior_depth, composite, j.depth_min, j.depth_max);
  if (cudaGetLastError() != cudaSuccess) return 21;
  CUDA_SYNC_AND_CHECK();
  CompositeInitNormalMap<<<g, b>>>(depth_map, normal_map, 0);
  if (cudaGetLastError() != cudaSuccess) return 22;
  CUDA_SYNC_AND_CHECK();
  return 0;
}

}  // namespace

extern "C" int ref_run(const RefJob* jp, RefOut* out) {
  const RefJob& j = *jp;
  if (j.N > MAX_NUM_SRC_IMAGE) return 1;
  // The reference's sweep with a prior (prior_depth_ncc) reads hypotheses[-1]
  // and M[-1] when FindMinCostWithin finds no hypothesis in the prior's band
  // (kernel_functions.cu:2431-2446, 2488-2493), before its local arrays; a test
  // process ended inside that run. Only the cost level (no iterations) is run.
  if (j.prior_mode == 1 && j.num_iterations > 0) return 31;
  Textures t;
  SetupTextures(j, t, true);
  const int W = j.W, H = j.H;
  BilateralWeightComputer weight_computer(j.sigma_s, j.sigma_c);
  // InitWorkspace, patch_match_cuda.cu:582-698.
  GpuMatPRNG rand_state(W, H);
  GpuMat<float> conf_map(W, H), depth_map(W, H), normal_map(W, H, 3);
  // Prior maps: InitPriorDepthAndNormalInfo (patch_match_cuda.cu:715-746) for
  // has_prior_depth; for propagate_depth the reference's sweep reads normal and
  // weight maps that stay 0 x 0 (:588-591), which the driver replaces by zero
  // maps of the image's size (the reading this library defines).
  const bool prior = j.prior_mode != 0;
  GpuMat<float> prior_depth(prior ? W : 0, prior ? H : 0, prior ? 1 : 0);
  GpuMat<float> prior_normal(prior ? W : 0, prior ? H : 0, prior ? 3 : 0);
  GpuMat<float> prior_wgt(prior ? W : 0, prior ? H : 0, prior ? 1 : 0);
  if (j.prior_mode == 1) {
    if (!j.init_depth || !j.init_normal) return 30;
    prior_depth.CopyToDevice(j.init_depth, W * sizeof(float));
    prior_normal.CopyToDevice(j.init_normal, W * sizeof(float));
    if (j.prior_wgt) prior_wgt.CopyToDevice(j.prior_wgt, W * sizeof(float));
    else ClearMap(prior_wgt);
  } else if (j.prior_mode == 2) {
    ClearMap(prior_normal);
    ClearMap(prior_wgt);
  }
  dim3 eb(THREADS_PER_BLOCK, THREADS_PER_BLOCK), eg((W - 1) / THREADS_PER_BLOCK + 1, (H - 1) / THREADS_PER_BLOCK + 1);
  // The reference launches InitDepthMap / InitNormalMap with 32x32 blocks
  // (patch_match_cuda.cu:93-100, 662-671). On sm_100a they need 96 / 72
  // registers per thread, so a 1024-thread block asks for more than the 64K
  // registers of an SM and the launch fails; CudaSyncAndCheck (cudacc.cc:50-64)
  // does not look at launch errors, so the reference continues with
  // uninitialised normals. The driver launches the same kernels with 32x16
  // blocks (the kernels index pixels from blockDim, so results are unchanged)
  // and checks every launch.
  dim3 ib(THREADS_PER_BLOCK, THREADS_PER_BLOCK / 2), ig((W - 1) / THREADS_PER_BLOCK + 1, (H - 1) / (THREADS_PER_BLOCK / 2) + 1);
  if (cudaGetLastError() != cudaSuccess) return 2;  // GpuMatPRNG's state initialisation
  if (!j.init_depth_random) {
    depth_map.CopyToDevice(j.init_depth, W * sizeof(float));
    normal_map.CopyToDevice(j.init_normal, W * sizeof(float));
    if (j.prior_mode == 2) {
      const int st = PropagateInit(j, t, rand_state, depth_map, normal_map, prior_depth);
      if (st) return st;
    }
    InitDepthMap<<<ig, ib>>>(depth_map, normal_map, rand_state, j.depth_min, j.depth_max, 0);
  } else {
    depth_map.FillWithRandomNumbers(j.depth_min, j.depth_max, rand_state);
    InitNormalMap<<<ig, ib>>>(normal_map, rand_state, 0);
  }
  if (cudaGetLastError() != cudaSuccess) return 3;
  CUDA_SYNC_AND_CHECK();
  GpuMat<float> cost_map(W, H, j.N);
  GpuMat<uint32_t> view_sel(W, H, 1);
  view_sel.FillWithScalar(0);
  GpuMat<float> grad_map(W, H);
  ComputeGradientMap<<<eg, eb>>>(grad_map, t.ref_tex);
  if (cudaGetLastError() != cudaSuccess) return 4;
  CUDA_SYNC_AND_CHECK();
  // Preprocess, patch_match_cuda.cu:448-491.
  t.sum_dev.reset(new CudaArrayWrapper<float>(W, H, 1));
  t.sum_dev->CopyFromGpuMat(*t.ref_image->sum_image);
  t.sum_tex = MakeArrayTexture(t.sum_dev->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);
  t.sqsum_dev.reset(new CudaArrayWrapper<float>(W, H, 1));
  t.sqsum_dev->CopyFromGpuMat(*t.ref_image->squared_sum_image);
  t.sqsum_tex = MakeArrayTexture(t.sqsum_dev->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);

  // SweepOptions, patch_match_cuda.cu:914-950.
  SweepOptions so;
  so.thread_index = 0;
  so.depth_min = j.depth_min;
  so.depth_max = j.depth_max;
  so.window_radius = j.R;
  so.window_step = j.S;
  so.sigma_spatial = j.sigma_s;
  so.sigma_color = j.sigma_c;
  so.geom_consistency_regularizer = j.geom_reg;
  so.geom_consistency_max_cost = j.geom_max;
  so.random_depth_ratio = j.rand_depth_ratio;
  so.random_angle1_range = j.a1;
  so.random_angle2_range = j.a2;
  so.init_ncc_matching_cost = j.init_mc;
  so.max_ncc_matching_cost = j.max_mc;
  so.alpha = j.alpha;
  so.beta = j.beta;
  so.num_good_hypothesis = j.good;
  so.num_bad_hypothesis = j.bad;
  so.thk = std::min(j.thk, j.N);
  so.num_samples = j.num_samples;
  so.geom_consistency = j.geom != 0;
  so.random_optimization = j.random_opt != 0;
  so.propagate_depth = j.prior_mode == 2;
  so.prior_depth_ncc = j.prior_mode == 1;

  const int BW = THREADS_PER_BLOCK, BH = THREADS_PER_BLOCK / 2;
  {  // InitConfMapKernel launch, patch_match_cuda.cu:963-981.
    dim3 b(BW, BH), g((W + BW - 1) / BW, (H + BH - 1) / BH);
    const int shared = (BH + j.R * 2) * (BW + j.R * 2) * sizeof(float);
    InitConfMapKernel<<<g, b, shared>>>(so, j.N, depth_map, normal_map, conf_map, cost_map, view_sel, prior_depth,
                                        prior_normal, prior_wgt, weight_computer, t.ref_tex, t.sum_tex, t.sqsum_tex,
                                        t.src_tex, t.src_depth_tex, t.poses_tex, 0);
    if (cudaGetLastError() != cudaSuccess) return 5;
    CUDA_SYNC_AND_CHECK();
  }
  {  // PropagationAndOptim, patch_match_cuda.cu:757-910.
    dim3 b(BW, BH), g((W + BW - 1) / BW, (H + BH - 1) / BH);
    const int shared = (BH * 2 + j.R * 2) * (BW + j.R * 2) * sizeof(float);
    for (int iter = 0; iter < j.num_iterations; ++iter) {
      so.th_mc = so.init_ncc_matching_cost * exp(-iter * iter / so.alpha);
      so.perturbation = 1.0f / std::pow(2.0f, iter);
      BlackPixelUpdateOpt<<<g, b, shared>>>(rand_state, depth_map, normal_map, conf_map, grad_map, cost_map, view_sel,
                                            prior_depth, prior_normal, prior_wgt, j.N, so, weight_computer, t.ref_tex,
                                            t.sum_tex, t.sqsum_tex, t.src_tex, t.src_depth_tex, t.poses_tex);
      CUDA_SYNC_AND_CHECK();
      RedPixelUpdateOpt<<<g, b, shared>>>(rand_state, depth_map, normal_map, conf_map, grad_map, cost_map, view_sel,
                                          prior_depth, prior_normal, prior_wgt, j.N, so, weight_computer, t.ref_tex,
                                          t.sum_tex, t.sqsum_tex, t.src_tex, t.src_depth_tex, t.poses_tex);
      if (cudaGetLastError() != cudaSuccess) return 6;
      CUDA_SYNC_AND_CHECK();
      if (j.local_opt && iter > 2 && j.prior_mode != 1) {  // patch_match_cuda.cu:861
        BlackPixelLocalOptimization<<<g, b, shared>>>(rand_state, depth_map, normal_map, conf_map, cost_map, view_sel,
                                                      j.N, so, weight_computer, t.ref_tex, t.sum_tex, t.sqsum_tex,
                                                      t.src_tex, t.src_depth_tex, t.poses_tex);
        CUDA_SYNC_AND_CHECK();
        RedPixelLocalOptimization<<<g, b, shared>>>(rand_state, depth_map, normal_map, conf_map, cost_map, view_sel,
                                                    j.N, so, weight_computer, t.ref_tex, t.sum_tex, t.sqsum_tex,
                                                    t.src_tex, t.src_depth_tex, t.poses_tex);
        if (cudaGetLastError() != cudaSuccess) return 7;
        CUDA_SYNC_AND_CHECK();
      }
    }
  }
  if (out->depth) depth_map.CopyToHost(out->depth, W * sizeof(float));
  if (out->normal) normal_map.CopyToHost(out->normal, W * sizeof(float));
  if (out->conf) conf_map.CopyToHost(out->conf, W * sizeof(float));
  if (out->cost) cost_map.CopyToHost(out->cost, W * sizeof(float));
  if (out->view_sel) view_sel.CopyToHost(out->view_sel, W * sizeof(uint32_t));
  CUDA_SYNC_AND_CHECK();
  return 0;
}

// The propagate-depth initial maps alone (before InitDepthMap draws random
// hypotheses for the pixels still without a depth): depth and normal hold the
// given maps on entry and the composited maps on return; prior receives the
// consistent medians.
extern "C" int ref_propagate_init(const RefJob* jp, float* depth, float* normal, float* prior) {
  const RefJob& j = *jp;
  if (j.N > MAX_NUM_SRC_IMAGE || !j.src_depth || !j.init_depth || !j.init_normal) return 1;
  Textures t;
  SetupTextures(j, t, false);
  GpuMatPRNG rand_state(j.W, j.H);
  if (cudaGetLastError() != cudaSuccess) return 2;
  GpuMat<float> depth_map(j.W, j.H), normal_map(j.W, j.H, 3), prior_depth(j.W, j.H);
  depth_map.CopyToDevice(j.init_depth, j.W * sizeof(float));
  normal_map.CopyToDevice(j.init_normal, j.W * sizeof(float));
  const int st = PropagateInit(j, t, rand_state, depth_map, normal_map, prior_depth);
  if (st) return st;
  depth_map.CopyToHost(depth, j.W * sizeof(float));
  normal_map.CopyToHost(normal, j.W * sizeof(float));
  prior_depth.CopyToHost(prior, j.W * sizeof(float));
  CUDA_SYNC_AND_CHECK();
  return 0;
}

// RunFilter(false), patch_match_cuda.cu:1075-1108.
extern "C" int ref_filter(const RefJob* jp, const float* depth_in, int min_consistent, float filter_max_cost,
                          float* depth_out) {
  const RefJob& j = *jp;
  if (j.N > MAX_NUM_SRC_IMAGE || !j.src_depth) return 1;
  Textures t;
  SetupTextures(j, t, false);
  GpuMat<float> depth_map(j.W, j.H);
  depth_map.CopyToDevice(depth_in, j.W * sizeof(float));
  dim3 eb(THREADS_PER_BLOCK, THREADS_PER_BLOCK);
  dim3 eg((j.W - 1) / THREADS_PER_BLOCK + 1, (j.H - 1) / THREADS_PER_BLOCK + 1);
  FilterDepthMapsKernel<<<eg, eb>>>(j.N, depth_map, j.geom_max, filter_max_cost, 0.02f, min_consistent, 0.5f,
                                    t.src_depth_tex, t.poses_tex, 0);
  if (cudaGetLastError() != cudaSuccess) return 8;
  CUDA_SYNC_AND_CHECK();
  depth_map.CopyToHost(depth_out, j.W * sizeof(float));
  return 0;
}

// ---------------------------------------------------------------------------
// Cross-view filter: CrossFilterCuda::Run and ::DedupRun
// (patch_match_cuda.cu:1139-1625) around the reference's CrossFilterKernel and
// DeduplicFilterKernel. The caller supplies the views' maps (the dedup inputs
// for ref_dedup, i.e. what ResetDepthMaps uploads), encoded normals and the
// per-problem pose records.
// ---------------------------------------------------------------------------
extern "C" {

struct RefCfView {
  int W, H;
  const float* depth;
  const uint32_t* code;  // may be NULL for ref_dedup
  int ref_flag;
};

struct RefCfProblem {
  int ref, num_src;
  const int* src;
  const float* poses;  // num_src * 43
  float refK[4], refiK[4];
};

}  // extern "C"

namespace {

template <typename T>
std::unique_ptr<CudaArrayWrapper<T>> Layered(int nv, const RefCfView* views, size_t max_w, size_t max_h,
                                             bool codes) {
  // InitDepthMaps / InitNormalMaps: every view padded to max_w x max_h with 0.
  std::vector<T> host(max_w * max_h * nv, T(0));
  for (int v = 0; v < nv; ++v) {
    const T* src = codes ? reinterpret_cast<const T*>(views[v].code) : reinterpret_cast<const T*>(views[v].depth);
    if (!src) continue;
    for (int r = 0; r < views[v].H; ++r)
      memcpy(host.data() + max_w * max_h * v + max_w * r, src + (size_t)r * views[v].W, sizeof(T) * views[v].W);
  }
  std::unique_ptr<CudaArrayWrapper<T>> dev(new CudaArrayWrapper<T>(max_w, max_h, nv));
  dev->CopyToDevice(host.data());
  return dev;
}

cudaTextureObject_t PosesTexture(const RefCfProblem& p, std::unique_ptr<CudaArrayWrapper<float>>& holder) {
  SetRefK(p.refK, 0);
  SetRefInvK(p.refiK, 0);
  holder.reset(new CudaArrayWrapper<float>(K_NUM_TFORM_PARAMS, p.num_src, 1));
  holder->CopyToDevice(p.poses);
  return MakeArrayTexture(holder->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);
}

}  // namespace

extern "C" int ref_cross_filter(int nv, const RefCfView* views, int np, const RefCfProblem* probs,
                                float filter_max_cost, float max_normal_error, float depth_diff, int min_consistent,
                                float* const* refined_out) {
  size_t max_w = 0, max_h = 0;
  for (int v = 0; v < nv; ++v) {
    max_w = std::max<size_t>(max_w, views[v].W);
    max_h = std::max<size_t>(max_h, views[v].H);
  }
  auto depth_dev = Layered<float>(nv, views, max_w, max_h, false);
  auto code_dev = Layered<unsigned int>(nv, views, max_w, max_h, true);
  cudaTextureObject_t depth_tex = MakeArrayTexture(depth_dev->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);
  cudaTextureObject_t code_tex = MakeArrayTexture(code_dev->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);
  int rc = 0;
  for (int k = 0; k < np && rc == 0; ++k) {
    const RefCfProblem& p = probs[k];
    if (p.num_src < 1) continue;  // :1504-1506
    if (p.num_src > MAX_NUM_CROSS_SRC) { rc = 1; break; }
    std::unique_ptr<CudaArrayWrapper<float>> poses_dev;
    cudaTextureObject_t poses_tex = PosesTexture(p, poses_dev);
    const int W = views[p.ref].W, H = views[p.ref].H;
    GpuMat<float> refined(W, H);
    CUDA_SAFE_CALL(cudaMemset2D(refined.GetPtr(), refined.GetPitch(), 0, W * sizeof(float), H));
    ImageIdxs idxs;
    memset(&idxs, 0, sizeof(idxs));
    idxs.list[0] = p.ref;
    for (int i = 0; i < p.num_src; ++i) idxs.list[i + 1] = p.src[i];
    idxs.length = p.num_src + 1;
    // 32x8 blocks over the padded size (the reference uses 32x32; every
    // thread is independent and indexes from blockDim).
    dim3 b(THREADS_PER_BLOCK, 8), g((max_w - 1) / THREADS_PER_BLOCK + 1, (max_h - 1) / 8 + 1);
    CrossFilterKernel<<<g, b>>>(p.num_src, W, H, 0.0f, filter_max_cost, max_normal_error, depth_diff,
                                std::min(min_consistent, p.num_src), idxs, refined, depth_tex, code_tex, poses_tex, 0);
    if (cudaGetLastError() != cudaSuccess) rc = 2;
    CUDA_SYNC_AND_CHECK();
    if (rc == 0) refined.CopyToHost(refined_out[p.ref], W * sizeof(float));
    cudaDestroyTextureObject(poses_tex);
  }
  cudaDestroyTextureObject(depth_tex);
  cudaDestroyTextureObject(code_tex);
  return rc;
}

extern "C" int ref_dedup(int nv, const RefCfView* views, int np, const RefCfProblem* probs, float filter_max_cost,
                         float depth_diff, int min_consistent, uint32_t* const* vis_out, float* const* delta_out) {
  size_t max_w = 0, max_h = 0;
  for (int v = 0; v < nv; ++v) {
    max_w = std::max<size_t>(max_w, views[v].W);
    max_h = std::max<size_t>(max_h, views[v].H);
  }
  auto depth_dev = Layered<float>(nv, views, max_w, max_h, false);
  cudaTextureObject_t depth_tex = MakeArrayTexture(depth_dev->GetPtr(), cudaFilterModePoint, cudaReadModeElementType);
  GpuMat<uint32_t> vis(max_w, max_h, nv);
  dim3 b(THREADS_PER_BLOCK, 8), g((max_w - 1) / THREADS_PER_BLOCK + 1, (max_h - 1) / 8 + 1);
  FillGpuMat<<<g, b>>>(max_w, max_h, vis);
  int rc = cudaGetLastError() != cudaSuccess ? 3 : 0;
  CUDA_SYNC_AND_CHECK();
  for (int k = 0; k < np && rc == 0; ++k) {
    const RefCfProblem& p = probs[k];
    if (p.num_src < 1) continue;  // :1568-1570
    if (p.num_src > MAX_NUM_CROSS_SRC) { rc = 1; break; }
    std::unique_ptr<CudaArrayWrapper<float>> poses_dev;
    cudaTextureObject_t poses_tex = PosesTexture(p, poses_dev);
    const int W = views[p.ref].W, H = views[p.ref].H;
    ImageLists lists;
    memset(&lists, 0, sizeof(lists));
    lists.list[0].id = p.ref;
    lists.list[0].flag = views[p.ref].ref_flag != 0;
    for (int i = 0; i < p.num_src; ++i) {
      lists.list[i + 1].id = p.src[i];
      lists.list[i + 1].flag = views[p.src[i]].ref_flag != 0;
    }
    lists.length = p.num_src + 1;
    GpuMat<float> delta(W, H);
    // The reference's FillWithScalar clears W*H*4 bytes of a pitched buffer
    // (gpu_mat.h:240-243), leaving later rows unset; clear all rows.
    CUDA_SAFE_CALL(cudaMemset2D(delta.GetPtr(), delta.GetPitch(), 0, W * sizeof(float), H));
    DeduplicFilterKernel<<<g, b>>>(p.num_src, W, H, filter_max_cost, depth_diff, std::min(min_consistent, p.num_src),
                                   lists, delta, vis, depth_tex, poses_tex, 0);
    if (cudaGetLastError() != cudaSuccess) rc = 2;
    CUDA_SYNC_AND_CHECK();
    if (rc == 0) delta.CopyToHost(delta_out[p.ref], W * sizeof(float));
    cudaDestroyTextureObject(poses_tex);
  }
  if (rc == 0) {
    std::vector<uint32_t> all(max_w * max_h * nv);
    vis.CopyToHost(all.data(), max_w * sizeof(uint32_t));
    for (int v = 0; v < nv; ++v)
      for (int r = 0; r < views[v].H; ++r)
        memcpy(vis_out[v] + (size_t)r * views[v].W, all.data() + max_w * max_h * v + max_w * r,
               sizeof(uint32_t) * views[v].W);
  }
  cudaDestroyTextureObject(depth_tex);
  return rc;
}
