// smvs_pool.cu — resident views, batched jobs and continuous admission.
//
// A pool keeps views (images as textures, optional depth/normal maps) resident
// in HBM under a byte budget with LRU eviction of unreferenced views, and runs
// many depth-map jobs (reference view + source views + options) together: one
// smvs_pool_step admits queued jobs while slots and memory allow, initialises
// them, then advances every active job by one PatchMatch iteration with one
// launch per checkerboard kernel for the whole batch (jobs of any size and
// source count; per-job parameters live in a device array), and retires the
// jobs that finished. The launch sequence of an unchanged batch is captured
// once into a CUDA graph and replayed. Jobs are independent: a job's maps are
// the same alone and in any mix (the RNG is keyed per job and pixel).
//
// No counterpart in the reference, which runs one PatchMatchACMMCuda per host
// thread and re-uploads every image for every reference view
// (patch_match_controller.cc:4330-4807, patch_match_cuda.cu:199-418).
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/smvs.h"
#include "smvs_device.cuh"
#include "smvs_kernels.h"

extern "C" void smvs_internal_set_error(const char* msg);
int smvs_internal_prepare_job(smvs::JobParams* p, const smvs_options* o);
void smvs_internal_pose_record(const smvs_view* ref, const smvs_view* src, float* out43);
cudaMemPool_t smvs_internal_device_pool(int device);

namespace {

// Device memory of views, kept maps and job state comes from the library's
// per-device stream-ordered memory pool, which keeps freed memory reserved:
// once a workload has run, admitting jobs and uploading views reuse that
// memory instead of calling the driver's allocator for every view and job
// (measured on the bench's batched passes: a device view upload 0.3 ms
// instead of 1-8 ms). A block is freed on the compute stream, after the last
// kernel that may read it; without a memory pool the plain allocator is used.
cudaError_t DevMalloc(cudaMemPool_t mem, cudaStream_t s, void** p, size_t bytes) {
  *p = nullptr;
  return mem ? cudaMallocFromPoolAsync(p, bytes, mem, s) : cudaMalloc(p, bytes);
}
void DevFree(cudaMemPool_t mem, cudaStream_t s, void* p) {
  if (!p) return;
  if (mem) cudaFreeAsync(p, s); else cudaFree(p);
}
// Texture-backed images: base and row pitch on 512-byte boundaries (the
// texture base alignment), the block allocated with room to align its start.
constexpr size_t kTexAlign = 512;
size_t AlignTex(size_t x) { return (x + kTexAlign - 1) & ~(kTexAlign - 1); }
cudaError_t DevMallocPitched(cudaMemPool_t mem, cudaStream_t s, void** base, void** p, size_t* pitch,
                             size_t row_bytes, int h) {
  *pitch = AlignTex(row_bytes);
  const cudaError_t e = DevMalloc(mem, s, base, *pitch * (size_t)h + kTexAlign);
  *p = e == cudaSuccess ? reinterpret_cast<void*>(AlignTex(reinterpret_cast<uintptr_t>(*base))) : nullptr;
  return e;
}

int Fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  smvs_internal_set_error(buf);
  return code;
}

#define POOL_CUDA(call)                                                                                    \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess) return Fail(SMVS_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

double NowSeconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t StorageBytes(int storage) { return storage == SMVS_STORE_U8 ? 1 : (storage == SMVS_STORE_F16 ? 2 : 4); }

cudaError_t MakeTexture(void* ptr, int fmt, int w, int h, size_t pitch, cudaTextureObject_t* tex) {
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = ptr;
  rd.res.pitch2D.width = (size_t)w;
  rd.res.pitch2D.height = (size_t)h;
  rd.res.pitch2D.pitchInBytes = pitch;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
  td.filterMode = cudaFilterModeLinear;
  td.normalizedCoords = 0;
  if (fmt == SMVS_STORE_U8) {
    rd.res.pitch2D.desc = cudaCreateChannelDesc<uint8_t>();
    td.readMode = cudaReadModeNormalizedFloat;
  } else if (fmt == SMVS_STORE_F16) {
    rd.res.pitch2D.desc = cudaCreateChannelDescHalf();
    td.readMode = cudaReadModeElementType;
  } else {
    rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
    td.readMode = cudaReadModeElementType;
  }
  return cudaCreateTextureObject(tex, &rd, &td, nullptr);
}

// Job state with a free list keyed by exact size: jobs of one workload have
// the same sizes, so steady-state admission reuses the pool's own blocks.
struct Arena {
  std::multimap<size_t, void*> free_blocks;
  size_t cached = 0;
  cudaMemPool_t mem = nullptr;
  cudaStream_t stream = nullptr;
  // A cached block of exactly `bytes`, or nullptr.
  void* Reuse(size_t bytes) {
    auto it = free_blocks.find(bytes);
    if (it == free_blocks.end()) return nullptr;
    void* p = it->second;
    free_blocks.erase(it);
    cached -= bytes;
    return p;
  }
  void* Get(size_t bytes) {
    void* p = nullptr;
    if (DevMalloc(mem, stream, &p, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      Trim();
      if (DevMalloc(mem, stream, &p, bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
      }
    }
    return p;
  }
  void Put(void* p, size_t bytes) {
    if (!p) return;
    free_blocks.emplace(bytes, p);
    cached += bytes;
  }
  void Trim() {  // stream-ordered: after every kernel already enqueued on `stream`
    for (auto& kv : free_blocks) DevFree(mem, stream, kv.second);
    free_blocks.clear();
    cached = 0;
  }
};

struct PoolView {
  int64_t id = 0;
  smvs_view meta;          // width/height/K/R/T/scale (pointers cleared)
  void* img = nullptr;     // storage-format pitched image
  void* img_block = nullptr;  // its allocation (img is its 512-byte aligned start)
  size_t pitch = 0;
  size_t img_bytes = 0;
  cudaTextureObject_t tex = 0;
  float* ref = nullptr;    // uint8-quantised normalised FP32 (as the reference view of a job)
  float* depth = nullptr;  // resident maps (optional)
  float* normal = nullptr;
  size_t dpitch = 0;
  float* depth_pitched = nullptr;
  void* depth_block = nullptr;  // allocation of depth_pitched
  cudaTextureObject_t dep_tex = 0;
  size_t map_bytes = 0;
  int refs = 0;            // queued + active jobs using this view
  uint64_t last_use = 0;
};

enum JobState { kQueued = 0, kActive = 1, kDone = 2, kFailed = 3 };

struct PoolJob {
  int64_t id = 0;
  smvs_options opt;
  int64_t ref = 0;
  std::vector<int64_t> srcs;
  int state = kQueued;
  int iter = 0;
  smvs::JobParams p;
  CUtensorMap map;         // the reference view's TMA descriptor (p.tma_box_w > 0)
  void* block = nullptr;   // one allocation for every per-job buffer
  size_t block_bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  cudaEvent_t done_ev = nullptr;  // recorded after the job's last iteration was enqueued
};

size_t Align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t JobBytes(int W, int H, int N) {
  const size_t WH = (size_t)W * H;
  return Align256(WH * 4) * 3            // ref_sum, ref_sqsum, grad
         + Align256((size_t)N * SMVS_POSE_FLOATS * 4)
         + Align256(WH * 4)              // depth
         + Align256(3 * WH * 4)          // normal
         + Align256(WH * 4)              // conf
         + Align256((size_t)N * WH * 4)  // cost
         + Align256(WH * 4);             // view_sel
}

}  // namespace

struct smvs_pool {
  smvs_pool_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::map<int64_t, PoolView> views;
  std::map<int64_t, PoolJob> jobs;
  std::deque<int64_t> queue;
  std::vector<int64_t> active;
  int64_t next_job = 1;
  uint64_t clock = 0;
  size_t bytes_used = 0;
  cudaMemPool_t mem = nullptr;  // the library's per-device memory pool (DevMalloc)
  Arena arena;
  // Batch arrays on the device and their pinned host staging (two sets, used
  // in turn, so that building a batch never waits for the previous upload).
  smvs::JobParams* d_jobs = nullptr;
  int* d_ints = nullptr;   // [iters (cap) | prefix (cap+32) | conf prefix (cap+32)]
  smvs::JobParams* h_jobs = nullptr;
  int* h_ints = nullptr;
  CUtensorMap* d_maps = nullptr;  // per job, as d_jobs
  CUtensorMap* h_maps = nullptr;
  smvs::JobParams* h_jobs_set[2] = {nullptr, nullptr};
  int* h_ints_set[2] = {nullptr, nullptr};
  CUtensorMap* h_maps_set[2] = {nullptr, nullptr};
  cudaEvent_t staged_ev[2] = {nullptr, nullptr};  // last upload from each set
  int cur_set = 0;
  int* d_status = nullptr;        // bounded waits of the kernels that gave up
  int* h_status = nullptr;        // pinned copy of d_status, refreshed after every step
  // Pose records of admitted jobs go through a pinned ring (no host sync).
  float* h_poses = nullptr;
  size_t poses_cap = 0, poses_off = 0;
  // Views uploaded from host memory: converted on copy_stream straight from
  // pinned staging slots (the compute stream waits for upload_ev before its
  // next launches), so uploads overlap the running iteration.
  cudaStream_t copy_stream = nullptr;
  struct Staging {
    void* host = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;
  };
  Staging staging[4];
  int staging_next = 0;
  cudaEvent_t upload_ev = nullptr;
  bool upload_pending = false;
  // Completion tracking without host synchronisation: jobs whose last
  // iteration is enqueued hold an event; the host keeps at most
  // kMaxStepsInFlight steps queued ahead of the GPU.
  std::vector<int64_t> finishing;
  std::deque<cudaEvent_t> step_events;
  std::vector<cudaEvent_t> free_events;
  cudaEvent_t GetEvent() {
    if (!free_events.empty()) {
      cudaEvent_t e = free_events.back();
      free_events.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
  }
  int capacity = 0;
  // Graph of the current batch's step (valid while the batch is unchanged).
  cudaGraphExec_t graph = nullptr;
  bool batch_dirty = true;
  std::vector<smvs::Batch> groups;
  int64_t launches = 0;
  int64_t graphs_built = 0;
  int64_t evictions = 0;
  int64_t steps = 0;

  ~smvs_pool() {
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& kv : jobs)
      if (kv.second.done_ev) cudaEventDestroy(kv.second.done_ev);
    for (cudaEvent_t e : step_events) cudaEventDestroy(e);
    for (cudaEvent_t e : free_events) cudaEventDestroy(e);
    for (int i = 0; i < 2; ++i) {
      if (staged_ev[i]) cudaEventDestroy(staged_ev[i]);
      if (h_jobs_set[i] != h_jobs) cudaFreeHost(h_jobs_set[i]);
      if (h_ints_set[i] != h_ints) cudaFreeHost(h_ints_set[i]);
      if (h_maps_set[i] != h_maps) cudaFreeHost(h_maps_set[i]);
    }
    for (auto& st : staging) {
      if (st.done) cudaEventDestroy(st.done);
      cudaFreeHost(st.host);
    }
    if (upload_ev) cudaEventDestroy(upload_ev);
    cudaFreeHost(h_status);
    cudaFreeHost(h_poses);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (auto& kv : jobs)
      if (kv.second.block) DevFree(mem, stream, kv.second.block);
    for (auto& kv : views) ReleaseView(kv.second);
    arena.Trim();
    cudaFree(d_jobs);
    cudaFree(d_ints);
    cudaFree(d_maps);
    cudaFree(d_status);
    cudaFreeHost(h_jobs);
    cudaFreeHost(h_ints);
    cudaFreeHost(h_maps);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
  // Callers make sure no kernel still reads the view (the streams are
  // synchronised); its memory goes back to the memory pool.
  void ReleaseView(PoolView& v) {
    if (v.tex) cudaDestroyTextureObject(v.tex);
    if (v.dep_tex) cudaDestroyTextureObject(v.dep_tex);
    DevFree(mem, stream, v.img_block);
    DevFree(mem, stream, v.ref);
    DevFree(mem, stream, v.depth_block);
    DevFree(mem, stream, v.depth);
    DevFree(mem, stream, v.normal);
    v = PoolView();
  }
  size_t ViewBytes(const PoolView& v) const { return v.img_bytes + v.map_bytes; }
  // Evict least recently used views that no job references until `need`
  // more bytes fit the budget. Returns false if it cannot.
  bool MakeRoom(size_t need) {
    while (bytes_used + need > opt.memory_budget_bytes) {
      int64_t victim = 0;
      uint64_t oldest = UINT64_MAX;
      for (auto& kv : views)
        if (kv.second.refs == 0 && kv.second.last_use < oldest) {
          oldest = kv.second.last_use;
          victim = kv.first;
        }
      if (oldest == UINT64_MAX) {
        // Cached free blocks count against the budget too: drop them first.
        if (arena.cached) {
          bytes_used -= arena.cached;
          arena.Trim();
          continue;
        }
        return false;
      }
      PoolView& v = views[victim];
      bytes_used -= ViewBytes(v);
      // Jobs that read the view may still be running (and an upload may still be
      // writing it): wait for both streams before its texture objects go.
      cudaStreamSynchronize(copy_stream);
      cudaStreamSynchronize(stream);
      ReleaseView(v);
      views.erase(victim);
      ++evictions;
    }
    return true;
  }
};

namespace {

// Batch integer arrays: iterations (cap) and two prefix arrays with one
// extra entry per group (at most kMaxGroups groups per batch).
constexpr int kMaxGroups = 32;
size_t IntsSize(int cap) { return (size_t)cap + 2 * ((size_t)cap + kMaxGroups); }

int EnsureCapacity(smvs_pool* P, int n) {
  if (n <= P->capacity) return SMVS_OK;
  int cap = P->capacity ? P->capacity : 16;
  while (cap < n) cap *= 2;
  cudaStreamSynchronize(P->stream);
  cudaFree(P->d_jobs);
  cudaFree(P->d_ints);
  cudaFree(P->d_maps);
  for (int i = 0; i < 2; ++i) {
    cudaFreeHost(P->h_jobs_set[i]);
    cudaFreeHost(P->h_ints_set[i]);
    cudaFreeHost(P->h_maps_set[i]);
    P->h_jobs_set[i] = nullptr; P->h_ints_set[i] = nullptr; P->h_maps_set[i] = nullptr;
  }
  P->d_jobs = nullptr; P->d_ints = nullptr; P->h_jobs = nullptr; P->h_ints = nullptr;
  P->d_maps = nullptr; P->h_maps = nullptr;
  POOL_CUDA(cudaMalloc(&P->d_jobs, sizeof(smvs::JobParams) * cap));
  POOL_CUDA(cudaMalloc(&P->d_ints, sizeof(int) * IntsSize(cap)));
  POOL_CUDA(cudaMalloc(&P->d_maps, sizeof(CUtensorMap) * cap));
  for (int i = 0; i < 2; ++i) {
    POOL_CUDA(cudaMallocHost(&P->h_jobs_set[i], sizeof(smvs::JobParams) * cap));
    POOL_CUDA(cudaMallocHost(&P->h_ints_set[i], sizeof(int) * IntsSize(cap)));
    POOL_CUDA(cudaMallocHost(&P->h_maps_set[i], sizeof(CUtensorMap) * cap));
  }
  P->h_jobs = P->h_jobs_set[P->cur_set];
  P->h_ints = P->h_ints_set[P->cur_set];
  P->h_maps = P->h_maps_set[P->cur_set];
  P->capacity = cap;
  P->batch_dirty = true;
  return SMVS_OK;
}

}  // namespace

extern "C" {

int smvs_pool_options_default(smvs_pool_options* o) {
  if (!o) return Fail(SMVS_EINVAL, "null options");
  memset(o, 0, sizeof(*o));
  o->memory_budget_bytes = (size_t)16 << 30;
  o->max_active_jobs = 64;
  o->image_storage = SMVS_STORE_U8;
  o->sweep_block_x = 32;
  o->use_graphs = 1;
  o->ref_tile_tma = 1;
  o->gpu_index = -1;
  o->sweep_threads_per_pixel = 1;
  return SMVS_OK;
}

int smvs_pool_create(const smvs_pool_options* o, void* stream, smvs_pool** out) {
  if (!o || !out) return Fail(SMVS_EINVAL, "null argument");
  *out = nullptr;
  if (o->max_active_jobs < 1) return Fail(SMVS_EINVAL, "max_active_jobs must be >= 1");
  if (o->image_storage < SMVS_STORE_U8 || o->image_storage > SMVS_STORE_F32) return Fail(SMVS_EINVAL, "bad image_storage");
  const int bx = o->sweep_block_x;
  if (bx != 8 && bx != 16 && bx != 32 && bx != 64) return Fail(SMVS_EINVAL, "sweep_block_x must be 8, 16, 32 or 64");
  const int tpp = o->sweep_threads_per_pixel;
  if (tpp != 1 && tpp != 2 && tpp != 4) return Fail(SMVS_EINVAL, "sweep_threads_per_pixel must be 1, 2 or 4");
  if (!smvs::ValidSweepShape(bx, tpp)) return Fail(SMVS_EINVAL, "sweep_block_x * sweep_threads_per_pixel must be <= 256");
  if (o->gpu_index >= 0) {
    cudaError_t e = cudaSetDevice(o->gpu_index);
    if (e != cudaSuccess) return Fail(SMVS_ECUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  }
  {
    const cudaError_t e = smvs::ConfigureKernels();
    if (e != cudaSuccess) return Fail(SMVS_ECUDA, "kernel set-up: %s", cudaGetErrorString(e));
  }
  auto* P = new smvs_pool();
  P->opt = *o;
  cudaGetDevice(&P->device);
  P->mem = smvs_internal_device_pool(P->device);
  if (stream) {
    P->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete P;
      return Fail(SMVS_ECUDA, "cudaStreamCreate failed");
    }
    P->own_stream = true;
  }
  P->arena.mem = P->mem;
  P->arena.stream = P->stream;
  int st = EnsureCapacity(P, o->max_active_jobs);
  if (st) { delete P; return st; }
  if (cudaMalloc(&P->d_status, sizeof(int)) != cudaSuccess ||
      cudaMemsetAsync(P->d_status, 0, sizeof(int), P->stream) != cudaSuccess ||
      cudaMallocHost(&P->h_status, sizeof(int)) != cudaSuccess) {
    delete P;
    return Fail(SMVS_ENOMEM, "pool status word");
  }
  *P->h_status = 0;
  P->poses_cap = (size_t)64 * 1024;
  if (cudaMallocHost(&P->h_poses, P->poses_cap * sizeof(float)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&P->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&P->upload_ev, cudaEventDisableTiming) != cudaSuccess) {
    delete P;
    return Fail(SMVS_ENOMEM, "pool staging");
  }
  *out = P;
  return SMVS_OK;
}

int smvs_pool_add_view(smvs_pool* P, int64_t view_id, const smvs_view* v, int memory) {
  if (!P || !v) return Fail(SMVS_EINVAL, "null argument");
  auto it = P->views.find(view_id);
  if (it != P->views.end()) {  // already resident: refresh its LRU position
    it->second.last_use = ++P->clock;
    return SMVS_OK;
  }
  if (v->width <= 0 || v->height <= 0 || !v->pixels) return Fail(SMVS_EINVAL, "view %lld: empty image", (long long)view_id);
  if (v->pixel_format != SMVS_PIX_U8 && v->pixel_format != SMVS_PIX_F32) return Fail(SMVS_EINVAL, "bad pixel format");
  if (v->K[0] == 0.f || v->K[4] == 0.f) return Fail(SMVS_EINVAL, "zero focal length");
  const int w = v->width, h = v->height;
  const size_t stride = v->row_stride ? v->row_stride : (size_t)w * (v->pixel_format == SMVS_PIX_U8 ? 1 : 4);
  const size_t need = (size_t)w * h * (StorageBytes(P->opt.image_storage) + 4) + 4096;
  if (!P->MakeRoom(need)) return Fail(SMVS_ENOMEM, "memory budget exhausted by views in use");
  PoolView pv;
  pv.id = view_id;
  pv.meta = *v;
  pv.meta.pixels = nullptr; pv.meta.depth = nullptr; pv.meta.normal = nullptr;
  // Allocated on the stream that writes the view: the compute stream for
  // device pixels, the copy stream for host pixels (the compute stream waits
  // for the copy stream's event before it reads them).
  cudaStream_t alloc_stream = memory == SMVS_MEM_DEVICE ? P->stream : P->copy_stream;
  cudaError_t e = DevMallocPitched(P->mem, alloc_stream, &pv.img_block, &pv.img, &pv.pitch,
                                   (size_t)w * StorageBytes(P->opt.image_storage), h);
  if (e == cudaSuccess) e = DevMalloc(P->mem, alloc_stream, (void**)&pv.ref, (size_t)w * h * 4);
  if (e == cudaSuccess && memory == SMVS_MEM_DEVICE) {
    // Device pixels: convert on the compute stream (ordered before every job).
    e = smvs::LaunchConvertImage(v->pixels, v->pixel_format, stride, w, h, pv.img, P->opt.image_storage, pv.pitch, 1,
                                 P->stream);
    if (e == cudaSuccess)
      e = smvs::LaunchConvertImage(v->pixels, v->pixel_format, stride, w, h, pv.ref, 3, (size_t)w * 4, 1, P->stream);
  } else if (e == cudaSuccess) {
    // Host pixels: copy them into a pinned staging slot (the caller's buffer
    // is only guaranteed during this call), then convert on the copy stream,
    // reading the slot over the bus, while the compute stream keeps running.
    smvs_pool::Staging& slot = P->staging[P->staging_next];
    P->staging_next = (P->staging_next + 1) % 4;
    if (slot.done) e = cudaEventSynchronize(slot.done);  // its previous upload has been converted
    if (e == cudaSuccess && slot.bytes < stride * h) {
      cudaFreeHost(slot.host);
      slot.host = nullptr;
      slot.bytes = 0;
      e = cudaHostAlloc(&slot.host, stride * h, cudaHostAllocMapped | cudaHostAllocPortable);
      if (e == cudaSuccess) slot.bytes = stride * h;
    }
    if (e == cudaSuccess && !slot.done) e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
    if (e == cudaSuccess) {
      memcpy(slot.host, v->pixels, stride * h);
      e = smvs::LaunchConvertImage(slot.host, v->pixel_format, stride, w, h, pv.img, P->opt.image_storage, pv.pitch,
                                   1, P->copy_stream);
    }
    if (e == cudaSuccess)
      e = smvs::LaunchConvertImage(slot.host, v->pixel_format, stride, w, h, pv.ref, 3, (size_t)w * 4, 1,
                                   P->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(slot.done, P->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(P->upload_ev, P->copy_stream);
    if (e == cudaSuccess) P->upload_pending = true;
  }
  if (e == cudaSuccess) e = MakeTexture(pv.img, P->opt.image_storage, w, h, pv.pitch, &pv.tex);
  if (e != cudaSuccess) {
    cudaStreamSynchronize(P->copy_stream);  // a conversion may still write the view
    P->ReleaseView(pv);
    return Fail(SMVS_ECUDA, "add_view: %s", cudaGetErrorString(e));
  }
  P->launches += 2;
  pv.img_bytes = pv.pitch * h + (size_t)w * h * 4;
  pv.last_use = ++P->clock;
  P->bytes_used += pv.img_bytes;
  P->views[view_id] = pv;
  return SMVS_OK;
}

int smvs_pool_has_view(smvs_pool* P, int64_t view_id, int* resident) {
  if (!P || !resident) return Fail(SMVS_EINVAL, "null argument");
  *resident = P->views.count(view_id) ? 1 : 0;
  return SMVS_OK;
}

static int SetMaps(smvs_pool* P, PoolView& v, const float* depth, const float* normal, int memory, bool device_src) {
  const int w = v.meta.width, h = v.meta.height;
  const size_t WH = (size_t)w * h;
  if (!v.depth) {
    const size_t need = WH * 4 * 4 + (size_t)w * 4 * h + 4096;
    if (!P->MakeRoom(need)) return Fail(SMVS_ENOMEM, "memory budget exhausted (view maps)");
    POOL_CUDA(DevMalloc(P->mem, P->stream, (void**)&v.depth, WH * 4));
    POOL_CUDA(DevMalloc(P->mem, P->stream, (void**)&v.normal, 3 * WH * 4));
    void* dp = nullptr;
    POOL_CUDA(DevMallocPitched(P->mem, P->stream, &v.depth_block, &dp, &v.dpitch, (size_t)w * 4, h));
    v.depth_pitched = static_cast<float*>(dp);
    POOL_CUDA(MakeTexture(v.depth_pitched, SMVS_STORE_F32, w, h, v.dpitch, &v.dep_tex));
    v.map_bytes = WH * 16 + v.dpitch * h;
    P->bytes_used += v.map_bytes;
  }
  const cudaMemcpyKind kind = (device_src || memory == SMVS_MEM_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  POOL_CUDA(cudaMemcpyAsync(v.depth, depth, WH * 4, kind, P->stream));
  if (normal) POOL_CUDA(cudaMemcpyAsync(v.normal, normal, 3 * WH * 4, kind, P->stream));
  POOL_CUDA(cudaMemcpy2DAsync(v.depth_pitched, v.dpitch, depth, (size_t)w * 4, (size_t)w * 4, h, kind, P->stream));
  if (kind == cudaMemcpyHostToDevice) POOL_CUDA(cudaStreamSynchronize(P->stream));
  P->batch_dirty = true;  // texture handles of jobs reading these maps are unchanged, but be safe
  return SMVS_OK;
}

int smvs_pool_set_view_maps(smvs_pool* P, int64_t view_id, const float* depth, const float* normal, int memory) {
  if (!P || !depth) return Fail(SMVS_EINVAL, "null argument");
  auto it = P->views.find(view_id);
  if (it == P->views.end()) return Fail(SMVS_EINVAL, "view %lld is not resident", (long long)view_id);
  it->second.last_use = ++P->clock;
  return SetMaps(P, it->second, depth, normal, memory, false);
}

int smvs_pool_submit(smvs_pool* P, const smvs_options* o, int64_t ref_id, const int64_t* src_ids, int n,
                     int64_t* job_id) {
  if (!P || !o || !src_ids || !job_id) return Fail(SMVS_EINVAL, "null argument");
  int st = smvs_options_check(o);
  if (st) return st;
  if (o->median_filter || o->conf_filter || o->est_curvature)
    return Fail(SMVS_EINVAL, "pool jobs do not run the median/confidence filters or curvature; use smvs_create");
  if (o->has_prior_depth || o->propagate_depth)
    return Fail(SMVS_EINVAL, "pool jobs do not take prior or propagated depth maps; use smvs_create");
  if (n < 1 || n > SMVS_MAX_SRC) return Fail(SMVS_EINVAL, "num_src=%d outside 1..%d", n, SMVS_MAX_SRC);
  auto rv = P->views.find(ref_id);
  if (rv == P->views.end()) return Fail(SMVS_EINVAL, "reference view %lld is not resident", (long long)ref_id);
  if (!o->init_depth_random && !rv->second.depth)
    return Fail(SMVS_EINVAL, "init_depth_random == 0 needs the reference view's maps (smvs_pool_set_view_maps)");
  for (int i = 0; i < n; ++i) {
    auto sv = P->views.find(src_ids[i]);
    if (sv == P->views.end()) return Fail(SMVS_EINVAL, "source view %lld is not resident", (long long)src_ids[i]);
    if (o->geom_consistency && !sv->second.depth)
      return Fail(SMVS_EINVAL, "geom_consistency needs source view %lld's depth map", (long long)src_ids[i]);
  }
  PoolJob J;
  J.id = P->next_job++;
  J.opt = *o;
  J.ref = ref_id;
  J.srcs.assign(src_ids, src_ids + n);
  J.t_submit = NowSeconds();
  rv->second.refs++;
  for (int i = 0; i < n; ++i) P->views[src_ids[i]].refs++;
  P->jobs[J.id] = J;
  P->queue.push_back(J.id);
  *job_id = J.id;
  return SMVS_OK;
}

namespace {

void CarveJob(PoolJob& J, int W, int H, int N) {
  const size_t WH = (size_t)W * H;
  char* b = static_cast<char*>(J.block);
  auto take = [&](size_t bytes) { char* p = b; b += Align256(bytes); return p; };
  smvs::JobParams& p = J.p;
  p.ref_sum = (const float*)take(WH * 4);
  p.ref_sqsum = (const float*)take(WH * 4);
  p.grad = (const float*)take(WH * 4);
  p.poses = (const float*)take((size_t)N * SMVS_POSE_FLOATS * 4);
  p.depth = (float*)take(WH * 4);
  p.normal = (float*)take(3 * WH * 4);
  p.conf = (float*)take(WH * 4);
  p.cost = (float*)take((size_t)N * WH * 4);
  p.view_sel = (uint32_t*)take(WH * 4);
}

// Build a job's parameters and initialise it (poses, reference moments,
// random or given-map initialisation). InitConf runs batched afterwards.
int Admit(smvs_pool* P, PoolJob& J) {
  PoolView& rv = P->views[J.ref];
  const smvs_options& o = J.opt;
  const int W = rv.meta.width, H = rv.meta.height, N = (int)J.srcs.size();
  smvs::JobParams& p = J.p;
  memset(&p, 0, sizeof(p));
  p.W = W; p.H = H; p.N = N; p.R = o.window_radius; p.S = o.window_step;
  const float ss = (float)o.sigma_spatial, sc = (float)o.sigma_color;
  p.sn = 1.0f / (2.0f * ss * ss);
  p.cn = 1.0f / (2.0f * sc * sc);
  p.depth_min = (float)o.depth_min;
  p.depth_max = (float)o.depth_max;
  p.rand_depth_ratio = o.random_depth_ratio;
  p.rand_a1 = o.random_angle1_range;
  p.rand_a2 = o.random_angle2_range;
  p.max_mc = (float)o.max_ncc_matching_cost;
  const float beta = (float)o.beta;
  p.inv_beta2 = 0.5f / (beta * beta);
  p.num_samples = o.num_samples;
  p.num_good = o.num_good_hypothesis;
  p.num_bad = o.num_bad_hypothesis;
  p.random_opt = o.random_optimization;
  p.geom = o.geom_consistency;
  p.thk = o.thk < N ? o.thk : N;
  p.geom_reg = (float)o.geom_consistency_regularizer;
  p.geom_max = (float)o.geom_consistency_max_cost;
  const float* K = rv.meta.K;
  p.refK[0] = K[0]; p.refK[1] = K[2]; p.refK[2] = K[4]; p.refK[3] = K[5];
  p.refiK[0] = 1.0f / p.refK[0];
  p.refiK[1] = -p.refK[1] / p.refK[0];
  p.refiK[2] = 1.0f / p.refK[2];
  p.refiK[3] = -p.refK[3] / p.refK[2];
  p.block_x = P->opt.sweep_block_x;
  p.tpp = P->opt.sweep_threads_per_pixel;
  p.ref = rv.ref;
  for (int i = 0; i < N; ++i) {
    PoolView& sv = P->views[J.srcs[i]];
    p.src_tex[i] = sv.tex;
    p.dep_tex[i] = sv.dep_tex;
    sv.last_use = ++P->clock;
  }
  rv.last_use = ++P->clock;
  {
    const int pst = smvs_internal_prepare_job(&p, &o);  // fits threads per pixel to N
    if (pst) return pst;
  }
  p.tma_box_w = p.tma_box_h = 0;
  memset(&J.map, 0, sizeof(J.map));
  if (P->opt.ref_tile_tma && smvs::EncodeRefMap(&J.map, p.ref, W, H, p.block_x, p.tpp, p.R)) {
    p.tma_box_w = smvs::RefTileW(p.block_x, p.R);
    p.tma_box_h = smvs::RefTileH(p.block_x, p.tpp, p.R);
  }
  J.block_bytes = JobBytes(W, H, N);
  J.block = P->arena.Reuse(J.block_bytes);  // cached blocks are already counted in bytes_used
  if (!J.block) {
    if (!P->MakeRoom(J.block_bytes)) return SMVS_ENOMEM;
    J.block = P->arena.Get(J.block_bytes);
    if (!J.block) return SMVS_ENOMEM;
    P->bytes_used += J.block_bytes;
  }
  CarveJob(J, W, H, N);
  const size_t nposes = (size_t)N * SMVS_POSE_FLOATS;
  if (P->poses_off + nposes > P->poses_cap) {
    // Ring wrap: every earlier record copy must have completed.
    POOL_CUDA(cudaStreamSynchronize(P->stream));
    P->poses_off = 0;
  }
  float* poses = P->h_poses + P->poses_off;
  P->poses_off += nposes;
  for (int i = 0; i < N; ++i)
    smvs_internal_pose_record(&rv.meta, &P->views[J.srcs[i]].meta, poses + (size_t)i * SMVS_POSE_FLOATS);
  POOL_CUDA(cudaMemcpyAsync((void*)p.poses, poses, nposes * 4, cudaMemcpyHostToDevice, P->stream));
  POOL_CUDA(smvs::LaunchPrepRef(p, (float*)p.ref_sum, (float*)p.ref_sqsum, (float*)p.grad, P->stream));
  if (!o.init_depth_random) {
    const size_t WH = (size_t)W * H;
    POOL_CUDA(cudaMemcpyAsync(p.depth, rv.depth, WH * 4, cudaMemcpyDeviceToDevice, P->stream));
    POOL_CUDA(cudaMemcpyAsync(p.normal, rv.normal, 3 * WH * 4, cudaMemcpyDeviceToDevice, P->stream));
  }
  p.stage_key = smvs::StageKey(o.random_seed, smvs::kStageInit);
  POOL_CUDA(smvs::LaunchInit(p, o.init_depth_random, (float)o.depth_min, (float)o.depth_max, P->stream));
  P->launches += 2;
  J.state = kActive;
  J.iter = 0;
  J.t_admit = NowSeconds();
  return SMVS_OK;
}

// Group jobs into batches sharing window, view bucket and launch shape; fill
// the pinned staging arrays at `offset` and record each group's batch.
int BuildGroups(smvs_pool* P, const std::vector<int64_t>& ids, std::vector<smvs::Batch>& groups) {
  groups.clear();
  if (ids.empty()) return SMVS_OK;
  // Use the other staging set; it may still feed the upload before last.
  P->cur_set ^= 1;
  if (P->staged_ev[P->cur_set]) POOL_CUDA(cudaEventSynchronize(P->staged_ev[P->cur_set]));
  P->h_jobs = P->h_jobs_set[P->cur_set];
  P->h_ints = P->h_ints_set[P->cur_set];
  P->h_maps = P->h_maps_set[P->cur_set];
  std::map<std::tuple<int, int, int, int, int>, std::vector<int64_t>> by_key;
  for (int64_t id : ids) {
    const smvs::JobParams& p = P->jobs[id].p;
    by_key[std::make_tuple(p.R, p.S, smvs::ViewBucket(p.N), p.block_x, p.tpp)].push_back(id);
  }
  int base = 0;
  const int cap = P->capacity;
  int* iters = P->h_ints;
  int* prefix = P->h_ints + cap;
  int* cprefix = P->h_ints + 2 * cap + kMaxGroups;
  // Groups are laid out one after another; prefix arrays of a group start at
  // its first job (each group's prefix restarts at 0 and has n+1 entries).
  int pos = 0;
  for (auto& kv : by_key) {
    const auto& list = kv.second;
    const int n = (int)list.size();
    smvs::Batch b{};
    b.R = std::get<0>(kv.first);
    b.S = std::get<1>(kv.first);
    b.NB = std::get<2>(kv.first);
    b.block_x = std::get<3>(kv.first);
    b.tpp = std::get<4>(kv.first);
    b.tma_polls = 0;
    b.tma_skip_copy = 0;
    b.persistent = P->opt.sweep_persistent != 0;
    b.grid_cap = smvs::PersistentGridCap();
    const int by = smvs::SweepRows(b.block_x, b.tpp);
    int tot = 0, ctot = 0;
    for (int k = 0; k < n; ++k) {
      PoolJob& J = P->jobs[list[k]];
      P->h_jobs[base + k] = J.p;
      P->h_maps[base + k] = J.map;
      iters[base + k] = J.iter;
      prefix[pos + k] = tot;
      cprefix[pos + k] = ctot;
      tot += J.p.blocks_x * ((J.p.H + by - 1) / by);
      ctot += J.p.conf_blocks_x * ((J.p.H + 7) / 8);
    }
    prefix[pos + n] = tot;
    cprefix[pos + n] = ctot;
    b.jobs = P->d_jobs + base;
    b.ref_maps = P->d_maps + base;
    b.status = P->d_status;
    b.iters = P->d_ints + base;
    b.block_start = P->d_ints + cap + pos;
    b.conf_block_start = P->d_ints + 2 * cap + kMaxGroups + pos;
    b.num_jobs = n;
    b.total_blocks = tot;
    b.total_conf_blocks = ctot;
    groups.push_back(b);
    base += n;
    pos += n + 1;
  }
  if ((int)groups.size() > kMaxGroups) return Fail(SMVS_EINVAL, "too many distinct job shapes in one batch");
  return SMVS_OK;
}

int Upload(smvs_pool* P, int njobs) {
  POOL_CUDA(cudaMemcpyAsync(P->d_jobs, P->h_jobs, sizeof(smvs::JobParams) * njobs, cudaMemcpyHostToDevice, P->stream));
  POOL_CUDA(cudaMemcpyAsync(P->d_maps, P->h_maps, sizeof(CUtensorMap) * njobs, cudaMemcpyHostToDevice, P->stream));
  POOL_CUDA(cudaMemcpyAsync(P->d_ints, P->h_ints, sizeof(int) * IntsSize(P->capacity), cudaMemcpyHostToDevice,
                            P->stream));
  if (!P->staged_ev[P->cur_set]) POOL_CUDA(cudaEventCreateWithFlags(&P->staged_ev[P->cur_set], cudaEventDisableTiming));
  POOL_CUDA(cudaEventRecord(P->staged_ev[P->cur_set], P->stream));
  return SMVS_OK;
}

// One iteration of every job of every group: black, red, [local black, red], advance.
int EnqueueIteration(smvs_pool* P, const std::vector<smvs::Batch>& groups) {
  for (const auto& b : groups) {
    for (int colour = 0; colour < 2; ++colour) POOL_CUDA(smvs::LaunchSweep(b, colour, P->stream));
    for (int colour = 0; colour < 2; ++colour) POOL_CUDA(smvs::LaunchLocalOpt(b, colour, P->stream));
    POOL_CUDA(smvs::LaunchAdvance(const_cast<int*>(b.iters), b.num_jobs, P->stream));
  }
  return SMVS_OK;
}

}  // namespace

// Retire finishing jobs whose last iteration has completed on the GPU (wait
// for them with `block`). A kernel's bounded wait that gave up shows in the
// status word copied back after every step.
static int PollFinishing(smvs_pool* P, bool block) {
  std::vector<int64_t> still;
  int st = SMVS_OK;
  for (int64_t id : P->finishing) {
    PoolJob& J = P->jobs[id];
    cudaError_t e = block ? cudaEventSynchronize(J.done_ev) : cudaEventQuery(J.done_ev);
    if (e == cudaErrorNotReady) {
      (void)cudaGetLastError();
      still.push_back(id);
      continue;
    }
    if (e != cudaSuccess) {
      st = Fail(SMVS_ECUDA, "pool step: %s", cudaGetErrorString(e));
      still.push_back(id);
      continue;
    }
    if (*P->h_status) st = Fail(SMVS_ETIMEDOUT, "a reference-tile copy did not complete; active jobs' maps are incomplete");
    P->free_events.push_back(J.done_ev);
    J.done_ev = nullptr;
    J.state = kDone;
    J.t_done = NowSeconds();
    P->views[J.ref].refs--;
    for (int64_t sid : J.srcs) P->views[sid].refs--;
  }
  P->finishing.swap(still);
  return st;
}

// Wait until `job` is no longer finishing (its maps are final).
static int SettleJob(smvs_pool* P, PoolJob& J) {
  if (!J.done_ev) return SMVS_OK;
  POOL_CUDA(cudaEventSynchronize(J.done_ev));
  return PollFinishing(P, false);
}

int smvs_pool_step(smvs_pool* P, smvs_pool_stats* stats) {
  if (!P) return Fail(SMVS_EINVAL, "null pool");
  cudaSetDevice(P->device);
  (void)cudaGetLastError();
  int pst = PollFinishing(P, false);
  if (pst) return pst;
  // Uploads of views from host memory run on the copy stream: the compute
  // stream's next launches wait for them.
  if (P->upload_pending) {
    POOL_CUDA(cudaStreamWaitEvent(P->stream, P->upload_ev, 0));
    P->upload_pending = false;
  }
  // 1. Admit queued jobs while slots and memory allow.
  std::vector<int64_t> admitted;
  while (!P->queue.empty() && (int)(P->active.size() + P->finishing.size()) < P->opt.max_active_jobs) {
    PoolJob& J = P->jobs[P->queue.front()];
    int st = Admit(P, J);
    if (st == SMVS_ENOMEM) {
      if (J.block) {  // counted in bytes_used; return it to the cache
        P->arena.Put(J.block, J.block_bytes);
        J.block = nullptr;
      }
      if (P->active.empty() && P->finishing.empty())
        return Fail(SMVS_ENOMEM, "job %lld does not fit the memory budget", (long long)J.id);
      break;  // wait for active jobs to finish
    }
    if (st) return st;
    P->queue.pop_front();
    admitted.push_back(J.id);
    P->active.push_back(J.id);
    P->batch_dirty = true;
  }
  // 2. InitConf of the newly admitted jobs (batched).
  if (!admitted.empty()) {
    std::vector<smvs::Batch> g;
    int st = BuildGroups(P, admitted, g);
    if (st) return st;
    if ((st = Upload(P, (int)admitted.size()))) return st;
    for (const auto& b : g) POOL_CUDA(smvs::LaunchInitConf(b, P->stream));
    P->launches += (int64_t)g.size();
    P->batch_dirty = true;
  }
  // 3. One iteration of every active job.
  if (!P->active.empty()) {
    if (P->batch_dirty) {
      int st = BuildGroups(P, P->active, P->groups);
      if (st) return st;
      if ((st = Upload(P, (int)P->active.size()))) return st;
      if (P->opt.use_graphs) {
        cudaGraph_t g = nullptr;
        POOL_CUDA(cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal));
        int est = EnqueueIteration(P, P->groups);
        cudaError_t ce = cudaStreamEndCapture(P->stream, &g);
        if (est) { if (g) cudaGraphDestroy(g); return est; }
        if (ce != cudaSuccess) return Fail(SMVS_ECUDA, "graph capture: %s", cudaGetErrorString(ce));
        // A batch that changed only in its parameters (the same groups, so the
        // same launch sequence) updates the executable graph in place; launches
        // already enqueued keep the parameters they were enqueued with. A
        // changed launch sequence instantiates a new one.
        if (P->graph) {
          cudaGraphExecUpdateResultInfo info;
          if (cudaGraphExecUpdate(P->graph, g, &info) != cudaSuccess) {
            (void)cudaGetLastError();  // the refused update, not an earlier error
            cudaGraphExecDestroy(P->graph);
            P->graph = nullptr;
          }
        }
        if (!P->graph) {
          ce = cudaGraphInstantiate(&P->graph, g, 0);
          if (ce != cudaSuccess) {
            cudaGraphDestroy(g);
            return Fail(SMVS_ECUDA, "graph instantiate: %s", cudaGetErrorString(ce));
          }
          P->graphs_built++;
        }
        cudaGraphDestroy(g);
      }
      P->batch_dirty = false;
    }
    if (P->graph) {
      POOL_CUDA(cudaGraphLaunch(P->graph, P->stream));
    } else {
      int st = EnqueueIteration(P, P->groups);
      if (st) return st;
    }
    P->launches += 5 * (int64_t)P->groups.size();
    POOL_CUDA(cudaMemcpyAsync(P->h_status, P->d_status, sizeof(int), cudaMemcpyDeviceToHost, P->stream));
    // 4. Jobs whose last iteration is now enqueued leave the batch; they are
    // done once the GPU has run it.
    std::vector<int64_t> still;
    for (int64_t id : P->active) {
      PoolJob& J = P->jobs[id];
      J.iter++;
      if (J.iter >= J.opt.num_iterations) {
        J.done_ev = P->GetEvent();
        POOL_CUDA(cudaEventRecord(J.done_ev, P->stream));
        P->finishing.push_back(id);
        P->batch_dirty = true;
      } else {
        still.push_back(id);
      }
    }
    P->active.swap(still);
    P->steps++;
    // Keep at most two steps queued ahead of the GPU.
    cudaEvent_t ev = P->GetEvent();
    POOL_CUDA(cudaEventRecord(ev, P->stream));
    P->step_events.push_back(ev);
    while (P->step_events.size() > 2) {
      POOL_CUDA(cudaEventSynchronize(P->step_events.front()));
      P->free_events.push_back(P->step_events.front());
      P->step_events.pop_front();
    }
  } else if (!P->finishing.empty()) {
    // Nothing to enqueue: wait for the oldest finishing job.
    POOL_CUDA(cudaEventSynchronize(P->jobs[P->finishing.front()].done_ev));
  }
  pst = PollFinishing(P, false);
  if (pst) return pst;
  if (stats) {
    stats->queued = (int)P->queue.size();
    stats->active = (int)(P->active.size() + P->finishing.size());
    int done = 0;
    for (auto& kv : P->jobs) done += kv.second.state == kDone;
    stats->done = done;
    stats->bytes_used = P->bytes_used;
    stats->bytes_budget = P->opt.memory_budget_bytes;
    stats->views_resident = (int)P->views.size();
    stats->launches = P->launches;
    stats->graphs_built = P->graphs_built;
    stats->evictions = P->evictions;
    stats->steps = P->steps;
  }
  return SMVS_OK;
}

int smvs_pool_job_state(smvs_pool* P, int64_t job_id, int* state, double* latency_s) {
  if (!P || !state) return Fail(SMVS_EINVAL, "null argument");
  auto it = P->jobs.find(job_id);
  if (it == P->jobs.end()) return Fail(SMVS_EINVAL, "unknown job %lld", (long long)job_id);
  if (it->second.done_ev) {
    const int st = PollFinishing(P, false);
    if (st) return st;
  }
  *state = it->second.state;
  if (latency_s) *latency_s = it->second.state == kDone ? it->second.t_done - it->second.t_submit : -1.0;
  return SMVS_OK;
}

int smvs_pool_wait(smvs_pool* P, int64_t job_id, double timeout_s, int* state) {
  if (!P) return Fail(SMVS_EINVAL, "null pool");
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    int s = 0;
    int st = smvs_pool_job_state(P, job_id, &s, nullptr);
    if (st) return st;
    if (state) *state = s;
    if (s == kDone || s == kFailed) return SMVS_OK;
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el >= timeout_s)
      return Fail(SMVS_ETIMEDOUT, "job %lld not done after %.3f s", (long long)job_id, timeout_s);
    if ((st = smvs_pool_step(P, nullptr))) return st;
  }
}

int smvs_pool_get_map(smvs_pool* P, int64_t job_id, int which, void* out) {
  if (!P || !out) return Fail(SMVS_EINVAL, "null argument");
  auto it = P->jobs.find(job_id);
  if (it == P->jobs.end()) return Fail(SMVS_EINVAL, "unknown job %lld", (long long)job_id);
  PoolJob& J = it->second;
  {
    const int st = SettleJob(P, J);
    if (st) return st;
  }
  if (J.state != kDone || !J.block) return Fail(SMVS_ESTATE, "job %lld has no results", (long long)job_id);
  const size_t WH = (size_t)J.p.W * J.p.H;
  const void* src = nullptr;
  size_t bytes = 0;
  switch (which) {
    case SMVS_MAP_DEPTH: src = J.p.depth; bytes = WH * 4; break;
    case SMVS_MAP_NORMAL: src = J.p.normal; bytes = 3 * WH * 4; break;
    case SMVS_MAP_CONF: src = J.p.conf; bytes = WH * 4; break;
    case SMVS_MAP_COST: src = J.p.cost; bytes = (size_t)J.p.N * WH * 4; break;
    case SMVS_MAP_VIEW_SEL: src = J.p.view_sel; bytes = WH * 4; break;
    default: return Fail(SMVS_EINVAL, "unknown map %d", which);
  }
  POOL_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDefault, P->stream));
  POOL_CUDA(cudaStreamSynchronize(P->stream));
  return SMVS_OK;
}

int smvs_pool_keep_maps(smvs_pool* P, int64_t job_id) {
  if (!P) return Fail(SMVS_EINVAL, "null pool");
  auto it = P->jobs.find(job_id);
  if (it == P->jobs.end()) return Fail(SMVS_EINVAL, "unknown job %lld", (long long)job_id);
  PoolJob& J = it->second;
  {
    const int st = SettleJob(P, J);
    if (st) return st;
  }
  if (J.state != kDone || !J.block) return Fail(SMVS_ESTATE, "job %lld has no results", (long long)job_id);
  auto vit = P->views.find(J.ref);
  if (vit == P->views.end()) return Fail(SMVS_ESTATE, "reference view of job %lld was evicted", (long long)job_id);
  return SetMaps(P, vit->second, J.p.depth, J.p.normal, SMVS_MEM_DEVICE, true);
}

int smvs_pool_release(smvs_pool* P, int64_t job_id) {
  if (!P) return Fail(SMVS_EINVAL, "null pool");
  auto it = P->jobs.find(job_id);
  if (it == P->jobs.end()) return Fail(SMVS_EINVAL, "unknown job %lld", (long long)job_id);
  PoolJob& J = it->second;
  {
    const int st = SettleJob(P, J);
    if (st) return st;
  }
  if (J.state == kActive) return Fail(SMVS_ESTATE, "job %lld is running", (long long)job_id);
  if (J.state == kQueued) {
    for (auto q = P->queue.begin(); q != P->queue.end(); ++q)
      if (*q == job_id) { P->queue.erase(q); break; }
    P->views[J.ref].refs--;
    for (int64_t s : J.srcs) P->views[s].refs--;
  }
  if (J.block) {
    // Its kernels have completed (SettleJob); copies enqueued from it since
    // (keep_maps) precede, in stream order, any kernel of a job that reuses it.
    P->arena.Put(J.block, J.block_bytes);  // kept as cached memory (still counted in bytes_used)
    J.block = nullptr;
  }
  P->jobs.erase(it);
  return SMVS_OK;
}

int smvs_pool_stats_get(smvs_pool* P, smvs_pool_stats* s) {
  if (!P || !s) return Fail(SMVS_EINVAL, "null argument");
  s->queued = (int)P->queue.size();
  s->active = (int)P->active.size();
  int done = 0;
  for (auto& kv : P->jobs) done += kv.second.state == kDone;
  s->done = done;
  s->bytes_used = P->bytes_used;
  s->bytes_budget = P->opt.memory_budget_bytes;
  s->views_resident = (int)P->views.size();
  s->launches = P->launches;
  s->graphs_built = P->graphs_built;
  s->evictions = P->evictions;
  s->steps = P->steps;
  return SMVS_OK;
}

void smvs_pool_destroy(smvs_pool* P) { delete P; }

}  // extern "C"
