/*
 * smvs.h — C ABI of the B200-native PatchMatch multi-view-stereo depth-map engine.
 *
 * This is the drop-in boundary for SenseMap's per-reference-view depth-map stage.
 * Each entry point replaces one member of the reference's C++ operator
 *   sensemap::mvs::PatchMatchACMMCuda (src/mvs/patch_match_cuda.h:154-203)
 * and its option/problem types (src/controllers/patch_match_options.h:42-353),
 * as cited beside each declaration. Conventions (all entry points):
 *   - every function returns an int status (SMVS_OK == 0) and never exits the
 *     process; smvs_last_error() gives a thread-local message for the last failure;
 *   - caller-owned host buffers, library-owned device memory;
 *   - no global per-thread constant slots: every engine carries its own
 *     parameter block, so any number of engines may share a GPU;
 *   - plain C types only (no CUDA or torch types); a CUDA stream is passed as
 *     an opaque void* (cudaStream_t), NULL meaning an engine-owned stream.
 */
#ifndef SMVS_H_
#define SMVS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMVS_ABI_VERSION 1
/* Hard cap on source views per reference view. The reference caps at 8
 * (MAX_NUM_SRC_IMAGE, src/mvs/kernel_functions.h:28); the view-selection
 * bitmask is a uint32 (kernel_functions.cu:2205), which bounds it at 32. */
#define SMVS_MAX_SRC 32
/* Number of floats in one source-view pose record:
 * [fx cx fy cy | R_rel(9) | T_rel(3) | C(3) | P(3x4) | P^-1(3x4)]
 * (K_NUM_TFORM_PARAMS, kernel_functions.h:31; layout patch_match_cuda.cu:516-559). */
#define SMVS_POSE_FLOATS 43

typedef enum smvs_status {
  SMVS_OK = 0,
  SMVS_EINVAL = 1,    /* bad argument or unsupported option combination */
  SMVS_ENOMEM = 2,    /* device or host allocation failed / budget exceeded */
  SMVS_ECUDA = 3,     /* a CUDA runtime call failed */
  SMVS_ESTATE = 4,    /* call out of order (e.g. get before run) */
  SMVS_EIO = 5,       /* file read/write failed */
  SMVS_ETIMEDOUT = 6, /* a bounded wait gave up */
  SMVS_ECANCELED = 7  /* job cancelled */
} smvs_status;

/* Pixel type of caller images (host or device). Grey values are 0..255 in both. */
typedef enum smvs_pixel_format {
  SMVS_PIX_U8 = 0,
  SMVS_PIX_F32 = 1
} smvs_pixel_format;

/* How source images are stored on the device and fetched by the cost kernels.
 * All three use hardware bilinear filtering with border (zero) addressing, the
 * sampling the reference uses (patch_match_cuda.cu:258-278). */
typedef enum smvs_image_storage {
  SMVS_STORE_U8 = 0,  /* 1 B/px, normalised read (the reference's own format) */
  SMVS_STORE_F16 = 1, /* 2 B/px, precision form: FP16 storage, FP32 accumulation */
  SMVS_STORE_F32 = 2  /* 4 B/px, plain FP32 path */
} smvs_image_storage;

typedef enum smvs_memory {
  SMVS_MEM_HOST = 0,
  SMVS_MEM_DEVICE = 1 /* pointers are device pointers on the engine's GPU */
} smvs_memory;

/* Mirrors the fields of PatchMatchOptions (patch_match_options.h:42-304) that the
 * depth-map path reads, with the reference's defaults (smvs_options_default). */
typedef struct smvs_options {
  double depth_min;                        /* :74 */
  double depth_max;                        /* :75 */
  int window_radius;                       /* :78 */
  int window_step;                         /* :85 */
  double sigma_spatial;                    /* :89 (reference default = window_radius) */
  double sigma_color;                      /* :90 */
  int num_samples;                         /* :93 */
  int num_iterations;                      /* :106 */
  int geom_consistency;                    /* :110 */
  double geom_consistency_regularizer;     /* :116 */
  double geom_consistency_max_cost;        /* :120 */
  int filter;                              /* :125 */
  int filter_min_num_consistent;           /* :135 */
  double filter_geom_consistency_max_cost; /* :139 */
  double max_normal_error;                 /* :141 (degrees; cross-view filter) */
  int init_depth_random;                   /* :164 */
  float random_depth_ratio;                /* :166 */
  float random_angle1_range;               /* :167 (radians) */
  float random_angle2_range;               /* :168 (radians) */
  double init_ncc_matching_cost;           /* :180 */
  double max_ncc_matching_cost;            /* :184 */
  double alpha;                            /* :187 */
  double beta;                             /* :190 */
  int thk;                                 /* :192 (1..4) */
  int num_good_hypothesis;                 /* :197 */
  int num_bad_hypothesis;                  /* :198 */
  int random_optimization;                 /* :68 */
  int local_optimization;                  /* :69 */
  int est_curvature;                       /* :71 */
  int median_filter;                       /* :248 */
  int conf_filter;                         /* :234 */
  float depth_diff_threshold;              /* :231 */
  float conf_threshold;                    /* :237 */
  int has_prior_depth;                     /* :250 — the reference view's given depth and
                                              normal maps (ref.depth, ref.normal) are a prior:
                                              costs are weighted by agreement with it
                                              (ComputeNCCWeightFromPrior, kernel_functions.cu:316-340),
                                              the first argmin of a sweep keeps to a band
                                              around it (:2431-2442) and local optimisation
                                              is off (patch_match_cuda.cu:861) */
  int propagate_depth;                     /* :288 — with init_depth_random == 0: pixels without a
                                              given depth start from the source views' depth maps
                                              projected into the reference view (src[i].depth; a
                                              source without one is skipped), the median of
                                              consistent projections becomes a prior depth, and
                                              normals are fitted to the result
                                              (patch_match_cuda.cu:603-659); excludes
                                              has_prior_depth and geom_consistency */
  /* ---- fields with no counterpart in the reference ---- */
  uint64_t random_seed;  /* seed of the counter-based RNG (replaces cuRAND XORWOW,
                            gpu_mat_prng.cu:10-37); results are a pure function of
                            (inputs, options, seed) */
  int image_storage;     /* smvs_image_storage */
  int gpu_index;         /* CUDA device ordinal; -1 = current device */
} smvs_options;

/* One view: image + calibration. K, R, T follow the reference's Image
 * accessors (src/mvs/image.h GetK/GetR/GetT): K row-major 3x3, (R, T) the
 * world-to-camera transform, x_cam = R x_world + T. */
typedef struct smvs_view {
  int width;
  int height;
  int pixel_format;     /* smvs_pixel_format */
  size_t row_stride;    /* bytes between rows of `pixels`; 0 = dense */
  const void* pixels;   /* grey image, 0..255 */
  float K[9];
  float R[9];
  float T[3];
  float scale;          /* Problem::src_image_scales (patch_match_options.h:317); 0 or 1 = none.
                           K is scaled by it (patch_match_cuda.cu:526-530); the caller
                           passes the image already resampled to the scaled size. */
  const float* depth;   /* optional W*H depth map of this view (geometric pass:
                           source views' maps; ref view: initial map when
                           init_depth_random == 0) */
  const float* normal;  /* optional 3*W*H planar normal map (ref view initial map) */
} smvs_view;

/* Mirrors Problem (patch_match_options.h:306-353) with the non-owning pointers
 * resolved to the views themselves. */
typedef struct smvs_problem {
  smvs_view ref;
  const smvs_view* src;  /* num_src entries */
  int num_src;           /* 1..SMVS_MAX_SRC */
  const uint8_t* ref_mask; /* optional W*H mask; depth is zeroed where 0
                              (MaskDepthMapKernel, kernel_functions.cu:3080-3093) */
  int memory;            /* smvs_memory of pixels/depth/normal/ref_mask/ref_prior_wgt */
  const float* ref_prior_wgt; /* optional W*H prior weights of the reference view
                              (Problem::prior_wgt_maps, patch_match_options.h:333; read
                              by has_prior_depth, InitPriorDepthAndNormalInfo
                              patch_match_cuda.cu:715-746); NULL = all 0 */
} smvs_problem;

typedef struct smvs_engine smvs_engine;

/* Device pointers to an engine's maps (valid until smvs_destroy). Layouts are
 * dense row-major; normal and cost are planar (slice-major), like GpuMat's
 * slices (src/util/gpu_mat.h:194-198) without the pitch. */
typedef struct smvs_device_maps {
  int width, height, num_src;
  float* depth;      /* W*H */
  float* normal;     /* 3*W*H */
  float* conf;       /* W*H */
  float* cost;       /* N*W*H */
  uint32_t* view_sel;/* W*H */
} smvs_device_maps;

/* Fill `opt` with the reference's defaults (PatchMatchOptions, patch_match_options.h:42-304). */
int smvs_options_default(smvs_options* opt);

/* Validate options like PatchMatchOptions::Check (patch_match_options.cc:75-101),
 * plus this engine's limits (supported window radius/step pairs, thk <= 4). */
int smvs_options_check(const smvs_options* opt);

/* Replaces PatchMatchACMMCuda::PatchMatchACMMCuda(options, problem)
 * (patch_match_cuda.cu:422-432): uploads the reference and source views,
 * builds the 43-float pose records (InitTransforms :493-580) and the
 * reference moments (InitRefImage :110-197). `stream` is a cudaStream_t or NULL. */
int smvs_create(const smvs_options* opt, const smvs_problem* prob, void* stream,
                smvs_engine** out);

/* Replaces PatchMatchACMMCuda::Run (patch_match_cuda.cu:748-1057): random or
 * given initialisation, InitConfMapKernel, num_iterations checkerboard
 * iterations with local optimisation, then the optional filters. Work is
 * enqueued on the engine's stream; the call does not wait for it. */
int smvs_run(smvs_engine* eng);

/* Replaces PatchMatchACMMCuda::RunFilter(dedup) (patch_match_cuda.cu:1075-1108):
 * the geometric-consistency filter of the reference view's depth map (the
 * problem's ref.depth) against the source views' depth maps. */
int smvs_run_filter(smvs_engine* eng, int deduplication);

/* Replace GetDepthMap / GetNormalMap / GetConfMap (patch_match_cuda.cu:47-54,440-446).
 * Copy to caller host buffers (synchronises the engine's stream). */
int smvs_get_depth_map(smvs_engine* eng, float* out);        /* W*H */
int smvs_get_normal_map(smvs_engine* eng, float* out);       /* 3*W*H planar */
int smvs_get_conf_map(smvs_engine* eng, float* out);         /* W*H */
int smvs_get_cost_map(smvs_engine* eng, float* out);         /* N*W*H planar */
int smvs_get_view_sel_map(smvs_engine* eng, uint32_t* out);  /* W*H */
/* Replaces GetCurvatureMap (patch_match_cuda.cu:444-446): 2*W*H planar uint16,
 * available when est_curvature && geom_consistency (ComputeCurvatureMap,
 * kernel_functions.cu:1603-1653). */
int smvs_get_curvature_map(smvs_engine* eng, uint16_t* out);

int smvs_get_size(const smvs_engine* eng, int* width, int* height, int* num_src);
int smvs_get_device_maps(const smvs_engine* eng, smvs_device_maps* out);
/* Block until the engine's queued work is done. */
int smvs_synchronize(smvs_engine* eng);
/* Number of kernel launches this engine has enqueued so far. */
int64_t smvs_launch_count(const smvs_engine* eng);

/* Kernel kinds for per-launch timing. No counterpart in the reference beyond
 * its stdout CudaTimer per iteration (patch_match_cuda.cu:776, 908, 1055). */
typedef enum smvs_kernel_kind {
  SMVS_KERNEL_CONVERT = 0,
  SMVS_KERNEL_PREP = 1,
  SMVS_KERNEL_INIT = 2,
  SMVS_KERNEL_INIT_CONF = 3,
  SMVS_KERNEL_SWEEP = 4,
  SMVS_KERNEL_LOCAL_OPT = 5,
  SMVS_KERNEL_MASK = 6,
  SMVS_KERNEL_FILTER = 7,
  SMVS_KERNEL_POST = 8   /* curvature, median and confidence filters */
} smvs_kernel_kind;
/* Launch-shape knobs of the checkerboard kernels (results do not depend on
 * them). No counterpart in the reference. */
typedef struct smvs_tuning {
  int sweep_block_x; /* pixels per block row: 8, 16, 32 (default) or 64 (each spans two
                        image columns of the checkerboard); a block is 256 threads */
  int ref_tile_tma;  /* 1 (default): stage the reference tile with a TMA load where the image
                        qualifies (rows a multiple of 16 bytes, image at least one tile);
                        0: plain loads */
  int threads_per_pixel; /* 1 (default), 2 or 4 threads share one pixel's NCC windows (1:
                            the pixel's state in registers and local memory; 2, 4: in
                            shared memory, the smallest value >= this whose shared memory
                            fits the view count is used). Maps do not depend on it. */
  int persistent;        /* threads_per_pixel 1: 1 = each checkerboard sweep launch is a
                            persistent grid (resident blocks per SM x SMs) whose blocks loop
                            over the tiles (the local optimisation keeps one block per tile);
                            0 (default) = one block per tile. Maps do not depend on it. */
} smvs_tuning;
int smvs_set_tuning(smvs_engine* eng, const smvs_tuning* tuning);
/* The launch shape in use and whether the last smvs_run staged its reference
 * tiles with TMA (ref_tile_tma = 1) or with plain loads (0). */
int smvs_get_tuning(const smvs_engine* eng, smvs_tuning* tuning);
/* Launch-shape autotuner: on a scratch engine for (opt, prob), times one
 * iteration's checkerboard sweep for every launch shape (sweep_block_x 8, 16,
 * 32, 64 x threads_per_pixel 1, 2, 4, with threads_per_pixel 1 both launch
 * forms of `persistent`, reference tiles by TMA where the image qualifies),
 * best of `repeats` (<= 0: 3), and writes the fastest to `best`. The
 * candidates and their ms per sweep launch go to tried/ms (up to `capacity`),
 * their number to num_tried. Maps do not depend on the choice. */
int smvs_autotune(const smvs_options* opt, const smvs_problem* prob, void* stream, int repeats, smvs_tuning* best,
                  smvs_tuning* tried, double* ms, int capacity, int* num_tried);
/* Record CUDA events around every subsequent launch of this engine. */
int smvs_set_profiling(smvs_engine* eng, int enable);
/* Number of timed launches of `kind` and their summed device time (ms); synchronises. */
int smvs_get_profile(smvs_engine* eng, int kind, int* count, double* total_ms);
void smvs_destroy(smvs_engine* eng);

/* ---- resident views, batched jobs, continuous admission ------------------ */
/* No counterpart in the reference (which runs one PatchMatchACMMCuda per host
 * thread and uploads every image again for every reference view,
 * patch_match_controller.cc:4330-4807). A pool keeps views resident in HBM
 * under a byte budget (least recently used views that no job references are
 * evicted), admits submitted jobs while slots and memory allow, and advances
 * every active job one PatchMatch iteration per smvs_pool_step with one launch
 * per checkerboard kernel for the whole batch (captured once in a CUDA graph
 * while the batch is unchanged). A job's maps do not depend on which other
 * jobs run with it. Not thread-safe: drive a pool from one thread. */
typedef struct smvs_pool smvs_pool;

typedef struct smvs_pool_options {
  size_t memory_budget_bytes; /* views + job state + cached blocks */
  int max_active_jobs;        /* slots */
  int image_storage;          /* smvs_image_storage of resident views */
  int sweep_block_x;          /* launch shape (smvs_tuning) */
  int use_graphs;             /* capture each batch's iteration in a CUDA graph */
  int gpu_index;              /* -1 = current device */
  int ref_tile_tma;           /* stage reference tiles with TMA where a view qualifies (smvs_tuning) */
  int sweep_threads_per_pixel; /* threads per pixel of the checkerboard kernels (smvs_tuning) */
  int sweep_persistent;        /* persistent checkerboard launches (smvs_tuning.persistent) */
} smvs_pool_options;

typedef struct smvs_pool_stats {
  int queued, active, done;
  size_t bytes_used, bytes_budget;
  int views_resident;
  int64_t launches, graphs_built, evictions, steps;
} smvs_pool_stats;

typedef enum smvs_job_state { SMVS_JOB_QUEUED = 0, SMVS_JOB_ACTIVE = 1, SMVS_JOB_DONE = 2, SMVS_JOB_FAILED = 3 } smvs_job_state;
typedef enum smvs_map_kind {
  SMVS_MAP_DEPTH = 0, SMVS_MAP_NORMAL = 1, SMVS_MAP_CONF = 2, SMVS_MAP_COST = 3, SMVS_MAP_VIEW_SEL = 4
} smvs_map_kind;

int smvs_pool_options_default(smvs_pool_options* opt);
int smvs_pool_create(const smvs_pool_options* opt, void* stream, smvs_pool** out);
/* Make a view resident (image only; K/R/T as in smvs_view). Re-adding a
 * resident id only refreshes its LRU position. `memory`: smvs_memory of pixels.
 * Host pixels are copied into a pinned staging slot before the call returns
 * and converted on the pool's copy stream, overlapping the running step. */
int smvs_pool_add_view(smvs_pool* pool, int64_t view_id, const smvs_view* view, int memory);
int smvs_pool_has_view(smvs_pool* pool, int64_t view_id, int* resident);
/* Resident depth (W*H) and normal (3*W*H, may be NULL) maps of a view: the
 * initial maps when it is a reference view with init_depth_random == 0, and
 * its geometric term when it is a source view of a geom_consistency job. */
int smvs_pool_set_view_maps(smvs_pool* pool, int64_t view_id, const float* depth, const float* normal, int memory);
/* Queue a job (photometric or geometric pass of one reference view). The
 * post-filters (median, confidence, curvature) and the mask are not run by
 * pool jobs (rejected with SMVS_EINVAL); use smvs_create for those. */
int smvs_pool_submit(smvs_pool* pool, const smvs_options* opt, int64_t ref_view, const int64_t* src_views,
                     int num_src, int64_t* job_id);
/* Admit, advance every active job one iteration, retire finished jobs. Does
 * not wait for the step's GPU work: a job whose last iteration has been
 * enqueued is done once the GPU has run it (smvs_pool_job_state polls; the map
 * getters wait), and the host stays at most two steps ahead of the GPU. A CUDA
 * error pending on the calling thread from earlier work is cleared first. */
int smvs_pool_step(smvs_pool* pool, smvs_pool_stats* stats);
/* smvs_job_state; latency_s (may be NULL) = completion - submission for done jobs, else -1. */
int smvs_pool_job_state(smvs_pool* pool, int64_t job_id, int* state, double* latency_s);
/* Step the pool until job `job_id` is done or failed, or `timeout_s` seconds
 * have passed (SMVS_ETIMEDOUT; the job keeps its place). *state (may be NULL)
 * receives the job's last state. The smvs_wait(job, timeout) of the serving
 * interface this library's pool provides; other jobs advance meanwhile. */
int smvs_pool_wait(smvs_pool* pool, int64_t job_id, double timeout_s, int* state);
/* Copy a done job's map (smvs_map_kind) to `out` (host or device). */
int smvs_pool_get_map(smvs_pool* pool, int64_t job_id, int which, void* out);
/* Store a done job's depth/normal as its reference view's resident maps. */
int smvs_pool_keep_maps(smvs_pool* pool, int64_t job_id);
/* Drop a queued or done job and return its memory to the pool's cache. */
int smvs_pool_release(smvs_pool* pool, int64_t job_id);
int smvs_pool_stats_get(smvs_pool* pool, smvs_pool_stats* stats);
void smvs_pool_destroy(smvs_pool* pool);

/* ---- no-allocation variant ----------------------------------------------- */
/* Largest number of source views smvs_filter_depth_map_noalloc accepts. */
#define SMVS_NOALLOC_MAX_SRC 32
/* The geometric-consistency filter of smvs_run_filter, for callers that cannot
 * allocate device memory: a serving process that reserved its whole device
 * budget at start-up and may not grow it per request, or a host whose
 * framework owns every device allocation. No counterpart in the reference. It
 * calls no cudaMalloc, cudaFree or other allocating routine: every input and
 * output is a caller-owned device buffer (prob->memory must be
 * SMVS_MEM_DEVICE; prob->ref.depth is the map to filter, each
 * prob->src[i].depth a source view's map, pixels are not read), and the
 * kernel's scratch — the pose records of at most SMVS_NOALLOC_MAX_SRC source
 * views, 5,504 bytes — lives in a fixed device array that every GPU loading
 * this library holds until the process exits. More source views are rejected
 * with SMVS_EINVAL, and the options pass smvs_options_check. The first call on
 * a device looks up that array's address (cudaGetSymbolAddress); make that
 * first call before any stream capture. All calls share the one array and each
 * call overwrites it (with a small kernel on `stream`) before its filter kernel
 * runs, so calls whose work overlaps on the GPU (different streams, or other
 * threads) race; serialise them. A CUDA error left pending on the calling
 * thread by earlier work is returned as SMVS_ECUDA (and thereby cleared)
 * before anything is enqueued. Work is enqueued on `stream` (NULL = the
 * default stream); `out_depth` is W*H floats. */
int smvs_filter_depth_map_noalloc(const smvs_options* opt, const smvs_problem* prob, float* out_depth,
                                  int deduplication, void* stream);

/* ---- cross-view filter and deduplication -------------------------------- */
/* CrossFilterCuda (src/mvs/patch_match_cuda.h:205-269, patch_match_cuda.cu:
 * 1111-1710): after every view of a cluster has a depth and normal map, each
 * problem's reference map is re-estimated as the median of the depths its
 * source views agree on (Run), then the cluster is deduplicated: a pixel seen
 * consistently by an earlier-processed view is dropped (DedupRun). The
 * controller drives it at patch_match_controller.cc:5575-6460.
 *
 * The set is the cluster's whole_ids / ref_flags (constructor arguments);
 * problems name views by their index in the set (the reference looks image ids
 * up in whole_ids, FindSrcImageIds :1427-1455). Run processes every problem in
 * one launch; DedupRun keeps the reference's sequential problem order wherever
 * two problems touch the same visibility layer and batches the rest. */

/* Most source views of one cross-filter problem (MAX_NUM_CROSS_SRC,
 * src/mvs/utils.h:39). */
#define SMVS_CROSS_MAX_SRC 31

/* One view of the set: an Image's size and K/R/T plus its DepthMap and
 * NormalMap (patch_match_cuda.cu:1139-1258). */
typedef struct smvs_filter_view {
  int width;
  int height;
  float K[9];
  float R[9];
  float T[3];
  const float* depth;   /* W*H */
  const float* normal;  /* 3*W*H planar; NULL when only dedup_run is used */
  int ref_flag;         /* ref_flags[i]: this view's dedup input is its refined map */
} smvs_filter_view;

/* One problem: Problem::ref_image_idx and src_image_extend_idxs
 * (patch_match_options.h:306-353), as indices into the view set. */
typedef struct smvs_filter_problem {
  int ref;
  const int* src;
  int num_src;          /* 0..SMVS_CROSS_MAX_SRC; 0 = skipped, as the reference does */
} smvs_filter_problem;

typedef struct smvs_cross_filter smvs_cross_filter;

/* CrossFilterCuda(options, problems, whole_ids, ref_flags) (:1111-1124) plus
 * InitDepthMaps/InitNormalMaps (:1139-1258): uploads every view's depth map and
 * its normal map as the kernel sees it (NormalMap::Encode, normal_map.cc:
 * 159-181, then the kernel's decode). Host maps (memory SMVS_MEM_HOST) are
 * copied before the call returns; device maps are read in stream order on
 * `stream`. Reads options depth_diff_threshold, filter_min_num_consistent,
 * filter_geom_consistency_max_cost, max_normal_error and gpu_index. Two
 * problems may not share a reference view; a view has fewer than 2^31 pixels.
 * Run, dedup_run and the device-map query only enqueue work; the host getters
 * wait for it. */
int smvs_cross_filter_create(const smvs_options* opt, const smvs_filter_view* views, int num_views,
                             const smvs_filter_problem* problems, int num_problems, int memory,
                             void* stream, smvs_cross_filter** out);
/* CrossFilterCuda::Run (:1493-1559), CrossFilterKernel (kernel_functions.cu:3561-3778). */
int smvs_cross_filter_run(smvs_cross_filter* cf);
/* CrossFilterCuda::DedupRun (:1561-1625), DeduplicFilterKernel
 * (kernel_functions.cu:3780-3916). Views with ref_flag read their refined map
 * (all zero if no problem refined them), the others their input map
 * (ResetDepthMaps :1260-1318). Needs filter_min_num_consistent >= 1. */
int smvs_cross_filter_dedup_run(smvs_cross_filter* cf);
/* GetRefineDepthMap (:1627-1639): W*H floats; SMVS_ESTATE unless run refined the view. */
int smvs_cross_filter_get_refined_depth_map(smvs_cross_filter* cf, int view, float* out);
/* GetDeduplicDepthMap (:1641-1664): the dedup input map where the view's
 * visibility keeps bit 31, else 0 (GetDeduplicDepthMapsLayer, kernel_functions.cu:3943-3960). */
int smvs_cross_filter_get_dedup_depth_map(smvs_cross_filter* cf, int view, float* out);
/* GetDeltDepthMap (:1666-1676): median |depth difference| / (threshold * depth)
 * per kept pixel; SMVS_ESTATE unless dedup_run processed the view as a reference. */
int smvs_cross_filter_get_delta_depth_map(smvs_cross_filter* cf, int view, float* out);
/* GetVisibilyMap (:1678-1704): bit 31 = kept, bit (30 - i) = consistent with source i. */
int smvs_cross_filter_get_visibility_map(smvs_cross_filter* cf, int view, uint32_t* out);
/* Device addresses of a view's maps (valid until destroy; NULL where absent). */
int smvs_cross_filter_get_device_maps(smvs_cross_filter* cf, int view, const float** refined,
                                      const float** delta, const uint32_t** visibility);
/* Kernel kinds of smvs_cross_filter_get_profile. */
typedef enum smvs_cross_filter_kernel {
  SMVS_CF_KERNEL_RUN = 0,    /* CrossFilterKernel, all problems */
  SMVS_CF_KERNEL_DEDUP = 1,  /* DeduplicFilterKernel, one launch per level */
  SMVS_CF_KERNEL_OTHER = 2   /* visibility fill, dedup depth maps */
} smvs_cross_filter_kernel;
/* Times every later launch with CUDA events on the filter's stream. */
int smvs_cross_filter_set_profiling(smvs_cross_filter* cf, int enable);
/* Timed launches of `kind` and their summed device time (ms); synchronises. */
int smvs_cross_filter_get_profile(smvs_cross_filter* cf, int kind, int* count, double* total_ms);
/* Number of kernels this filter launched so far. */
int64_t smvs_cross_filter_launch_count(smvs_cross_filter* cf);
/* Number of sequential dedup passes (launches) the last dedup_run needed. */
int smvs_cross_filter_dedup_levels(smvs_cross_filter* cf);
int smvs_cross_filter_synchronize(smvs_cross_filter* cf);
void smvs_cross_filter_destroy(smvs_cross_filter* cf);
/* Cross filters, depth-map pools (views, kept maps, job state), fusion and
 * the initial-map builders allocate from a per-device stream-ordered memory
 * pool that keeps freed memory reserved for the next call; this returns the
 * free part of it to the device (synchronises the device). gpu_index -1 =
 * current device. */
int smvs_cross_filter_release_cache(int gpu_index);

/* ---- initial depth/normal maps from the model ---------------------------- */
/* The maps PatchMatchController builds for a view before a PatchMatch pass
 * with init_depth_random == 0 (patch_match_controller.cc:4376-4460), as GPU
 * scatters with the reference's depth tests (results do not depend on the
 * order of points or faces). `view` supplies width, height, K, R and T (pixels
 * are not read). Outputs: depth W*H (0 where nothing landed), normal 3*W*H
 * planar (0 where nothing landed), and optionally depth_range[2], the pair
 * the reference returns (first = 1e-6, second = 1.1 x the largest depth
 * written, or 110 when nothing was). `memory` says where every array lives;
 * with SMVS_MEM_DEVICE and depth_range NULL the call only enqueues work on
 * `stream`, otherwise it waits for it. */
/* InitDepthMap (:1205-1307) + InitDepthMapFromSparsePoint (:483-518): `xyz`
 * are the sparse points whose track contains the view (n x 3 float); each
 * lands in a 7x7 window at its truncated pixel, nearest depth kept, normal 0. */
int smvs_init_depth_from_sparse_points(const smvs_view* view, const float* xyz, size_t num_points, int memory,
                                       float* depth, float* normal, float* depth_range, void* stream);
/* InitDepthMap with init_from_delaunay (:1205-1307, :1290-1291) +
 * InitDepthMapFromDelaunay (:398-474): the same sparse points, each at its
 * truncated pixel (a repeated pixel keeps its first point, as CGAL keeps the
 * first vertex at a position), are triangulated (2-D Delaunay over the pixel
 * positions, on the host) and every triangle's plane through its three
 * back-projected points is written to the pixels inside it: depth and the
 * camera-frame unit normal. A pixel on an edge shared by two triangles takes
 * the triangle with the largest vertex indices (the reference takes the later
 * face in CGAL's face order); on four co-circular points the triangulation's
 * diagonal may differ from CGAL's. At most 2^21 - 1 points. */
int smvs_init_depth_from_delaunay(const smvs_view* view, const float* xyz, size_t num_points, int memory,
                                  float* depth, float* normal, float* depth_range, void* stream);
/* Model2Depth (:520-642): TriangleMesh vertices_ (n x 3 double), faces_
 * (m x 3 int32) and face_normals_ (m x 3 double), rasterised with back-face
 * and field-of-view culling; normals are the camera-frame face normals. */
int smvs_init_depth_from_mesh(const smvs_view* view, const double* vertices, size_t num_vertices,
                              const int32_t* faces, size_t num_faces, const double* face_normals, int memory,
                              float* depth, float* normal, float* depth_range, void* stream);
/* Ply2Depth (:643-750): oriented dense points (PlyPoint x/y/z and nx/ny/nz as
 * two n x 3 float arrays) splatted into the odd pixels of a window of
 * 2^level pixels around each (level = PLY_INIT_DEPTH_LEVEL = 2, utils.h:40). */
int smvs_init_depth_from_dense_points(const smvs_view* view, const float* xyz, const float* normals,
                                      size_t num_points, int level, int memory, float* depth, float* normal,
                                      float* depth_range, void* stream);

/* ---- coarse-to-fine pyramid --------------------------------------------- */
/* Size of pyramid level `level` of a width x height image: the factor
 * 1 / 2^level, but never below 320 pixels on the longer side, and the rounded
 * sizes (PatchMatchController::ProcessProblem, patch_match_controller.cc:
 * 4407-4410; Image::Rescale, src/mvs/image.cc:51-52). `factor` may be NULL. */
int smvs_pyramid_level_size(int width, int height, int level, int* out_width, int* out_height, float* factor);
/* Image::Rescale / Bitmap::Rescale (src/mvs/image.cc:44-70, src/util/bitmap.cc:
 * 705-708, FreeImage's bilinear filter) on the device: a grey float image
 * (0..255) resampled to out_width x out_height with the triangle filter
 * widened by the inverse scale, rounded to integer grey levels. Device
 * buffers: `in` width*height, `out` out_width*out_height, `scratch`
 * out_width*height floats. Enqueued on `stream`. The caller scales K by the
 * size ratios as Image::Rescale does (image.cc:58-63). */
int smvs_rescale_image(const float* in, int width, int height, float* out, int out_width, int out_height,
                       void* scratch, void* stream);
/* DepthMap::Rescale and NormalMap::Rescale (src/mvs/depth_map.cc:32-55,
 * src/mvs/normal_map.cc:27-72: InterpolateImage -> ResampleImageBilinear,
 * src/util/mat.cc:18-58, then the normals re-normalised) on the device, to
 * out_width x out_height. Device buffers; `normal`/`out_normal` are planar
 * 3 x H x W and may be NULL, as may depth/out_depth (one of the two pairs must
 * be given). Enqueued on `stream`. */
int smvs_resample_maps(const float* depth, const float* normal, int width, int height, float* out_depth,
                       float* out_normal, int out_width, int out_height, void* stream);

/* ---- view selection and depth ranges from the sparse model (host) -------- */
/* One image of mvs::Model (src/mvs/model.h): the world-to-camera pose and
 * Image::IsRig. */
typedef struct smvs_model_image {
  float R[9];
  float T[3];
  int is_rig;
} smvs_model_image;

/* Model::GetMaxOverlappingImages (src/mvs/model.cc:701-935): for every image in
 * `candidates` (the reference's unique_image_idxs), the source views sharing the
 * most sparse points whose 75th-percentile triangulation angle reaches
 * min_triangulation_angle (degrees), best first (a shared point counts 1.5x
 * between images of the same rig kind); an image that observes no point falls
 * back to spatial neighbours (distance and viewing-angle score). Points are
 * Model::Point x/y/z (n x 3 float) with their tracks in CSR form
 * (track_offsets[n + 1], track_images). Output in CSR form: out_offsets
 * [num_images + 1] and out_images (capacity num_images * max_num_images); images
 * outside `candidates` get no list. Ties keep ascending image order (the
 * reference leaves their order unspecified). Host only; all host threads. */
int smvs_select_views(const smvs_model_image* images, int num_images, const float* points, size_t num_points,
                      const int32_t* track_offsets, const int32_t* track_images, const int32_t* candidates,
                      int num_candidates, int max_num_images, double min_triangulation_angle,
                      int32_t* out_offsets, int32_t* out_images);
/* Model::ComputeDepthRanges (:941-959): per image the depth range of the
 * model's bounding box corners (lt, rb as BoundingBox), first clamped to
 * >= 1e-6. ranges is num_images x 2. Host only. */
int smvs_compute_depth_ranges(const smvs_model_image* images, int num_images, const float bbox_lt[3],
                              const float bbox_rb[3], float* ranges);

/* ---- fusion of depth maps into a point cloud ----------------------------- */
/* StereoFusion (src/mvs/fusion.h:43-280, fusion.cc:648-2182): the image loop of
 * Run (:1160-1215), FuseImage (:1730-1792) and Fuse (:1794-2182). Images are
 * fused one after another in FindNextImage order (:697-727); in each image every
 * seed pixel that is not yet fused starts a depth-first traversal over the
 * overlapping images' pixels that agree with it in reprojection, depth and
 * normal, and a cluster with enough pixels and images becomes one point (the
 * medians of its pixels). Results are those of the reference run with one
 * fusion thread per image slice taking its seeds in order (num_slices slices,
 * one after another); the reference's concurrent slices race on the shared
 * pixel masks and have no single result. */
typedef struct smvs_fusion_options {
  int step_size;               /* seed stride in rows and columns (1) */
  int min_num_pixels;          /* >= 2 (5) */
  int max_num_pixels;          /* (10000) */
  int min_num_visible_images;  /* (3) */
  int max_traversal_depth;     /* > 0 (100) */
  double max_reproj_error;     /* pixels (2) */
  double max_depth_error;      /* relative (0.01f) */
  double max_normal_error;     /* degrees (10) */
  int with_normal;             /* (1) */
  int num_slices;              /* FuseImage's row slices, taken in order (1) */
  int gpu_index;               /* (0) */
} smvs_fusion_options;

/* One image: size, K/R/T (mvs::Image) and its maps. A view without a depth
 * map is not used (Run's Init, fusion.cc:979-990). */
typedef struct smvs_fusion_view {
  int width;
  int height;
  float K[9];
  float R[9];
  float T[3];
  const float* depth;    /* W*H; NULL = image not used */
  const float* normal;   /* 3*W*H planar (world normals are R^T n); needed with with_normal */
  const uint8_t* color;  /* W*H*3 interleaved RGB (Bitmap::GetPixel); NULL reads black */
  int is_rig;            /* Image::IsRig: FindNextImage prefers other images */
} smvs_fusion_view;

/* PlyPoint x/y/z, nx/ny/nz, r/g/b plus the point's score (fused_points_score_). */
typedef struct smvs_fused_point {
  float x, y, z;
  float nx, ny, nz;   /* 0 without with_normal */
  uint8_t r, g, b, pad;
  float score;
} smvs_fused_point;

typedef struct smvs_fusion smvs_fusion;

int smvs_fusion_options_default(smvs_fusion_options* opt);
/* StereoFusion(options, ...) with the maps and the overlapping image lists
 * (overlapping_images_, from Model::GetMaxOverlappingImages; CSR form
 * overlap_offsets[num_views + 1], overlap_images) given directly. `memory` says
 * where depth/normal/color live; host maps are copied before the call returns.
 * The views together hold fewer than 2^31 pixels. */
int smvs_fusion_create(const smvs_fusion_options* opt, const smvs_fusion_view* views, int num_views,
                       const int32_t* overlap_offsets, const int32_t* overlap_images, int memory, void* stream,
                       smvs_fusion** out);
/* Fuses every used image (Run :1160-1215). Enqueues the work on the stream
 * and waits for it. May be called once. */
int smvs_fusion_run(smvs_fusion* f);
/* Number of fused points and of visibility entries. */
int smvs_fusion_get_sizes(smvs_fusion* f, size_t* num_points, size_t* num_visibility);
/* GetFusedPoints / GetFusedPointsVisibility (:665-672) in the order the points
 * were fused: points[num_points], visibility offsets[num_points + 1] and image
 * indices, each point's images in ascending order (the reference lists them in
 * std::unordered_set order). Any output may be NULL. */
int smvs_fusion_get_points(smvs_fusion* f, smvs_fused_point* points, uint64_t* vis_offsets,
                           uint32_t* vis_images);
/* Device addresses of the same arrays (valid until destroy). */
int smvs_fusion_get_device_points(smvs_fusion* f, const smvs_fused_point** points, const uint64_t** vis_offsets,
                                  const uint32_t** vis_images);
/* StereoFusion::RemoveDuplicatePoints (fusion.cc:2184-2266; Run calls it after
 * the image loop when Options::remove_duplicate_pnts, the default, fusion.cc:
 * 1271-1274): in fusion order each point claims the pixel it projects to in each
 * of its images; a point that meets an occupant seen by more images is dropped
 * (and visits no further image), otherwise it takes the pixel and the occupant
 * is dropped. A point's images are visited in ascending order (the reference
 * iterates its std::unordered_set). The cloud is compacted in place (order kept);
 * *num_removed (may be NULL) receives the number of points dropped. */
int smvs_fusion_remove_duplicate_points(smvs_fusion* f, size_t* num_removed);
/* StereoFusion::RemoveOutliers (fusion.cc:2542-2611; Run calls it when
 * Options::outlier_removal, off by default, :1277-1279) with the spacing of
 * ComputeAverageDistance (patch_match_controller.cc:115-228): each point's mean
 * distance to its nb_neighbors nearest points (exact k-nearest neighbours on the
 * GPU) is blended into its score as score * 0.6 + spacing / (max_spacing_factor *
 * mean spacing) * 0.4, the scores are histogrammed over 256 bins between their
 * minimum and maximum, and points in a bin holding under 1 % of the cloud whose
 * cumulative share is at least 90 % are dropped. Scores are updated in place. */
int smvs_fusion_remove_outliers(smvs_fusion* f, int nb_neighbors, double max_spacing_factor, size_t* num_removed);
/* The images in the order they were fused (count <= num_views). */
int smvs_fusion_get_image_order(smvs_fusion* f, int* order, int* count);
/* fused_pixel_masks_ of a view after run: W*H bytes, 1 = fused. */
int smvs_fusion_get_mask(smvs_fusion* f, int view, uint8_t* out);
/* Kernel kinds of smvs_fusion_get_profile. */
typedef enum smvs_fusion_kernel {
  SMVS_FUSION_KERNEL_CLOSURE = 0,  /* candidate clusters of every seed of an image */
  SMVS_FUSION_KERNEL_ORDER = 1,    /* claim lists, predecessors and the replay order */
  SMVS_FUSION_KERNEL_REPLAY = 2,   /* the seeds' traversals in dependency order */
  SMVS_FUSION_KERNEL_OTHER = 3     /* point maps, output compaction */
} smvs_fusion_kernel;
int smvs_fusion_set_profiling(smvs_fusion* f, int enable);
int smvs_fusion_get_profile(smvs_fusion* f, int kind, int* count, double* total_ms);
int64_t smvs_fusion_launch_count(smvs_fusion* f);
void smvs_fusion_destroy(smvs_fusion* f);

/* Thread-local message describing the last failure on this thread. */
const char* smvs_last_error(void);

/* ---- on-disk formats (host only) ---------------------------------------- */
/* Mat<T>::Write / Read (src/util/mat.h:179-215): text header "W&H&D&" followed by
 * the little-endian payload, slice-major then row-major. */
int smvs_write_mat_f32(const char* path, const float* data, int width, int height, int depth);
int smvs_write_mat_u32(const char* path, const uint32_t* data, int width, int height, int depth);
int smvs_write_mat_u16(const char* path, const uint16_t* data, int width, int height, int depth);
/* Reads the header; if `data` is NULL only the sizes are returned. `elem_size` is 2 or 4. */
int smvs_read_mat(const char* path, void* data, size_t capacity_bytes, int elem_size,
                  int* width, int* height, int* depth);
/* NormalMap::Encode / Decode (src/mvs/normal_map.cc:109-181): one uint32 per pixel. */
int smvs_encode_normal_map(const float* normal, int width, int height, uint32_t* code);
int smvs_decode_normal_map(const uint32_t* code, int width, int height, float* normal);
/* DepthMap::Write + NormalMap::Write + Mat<float>::Write of the conf map into
 * <dir>/{depth_maps,normal_maps,conf_maps}/<image_name>.<type>.bin
 * (base/common.h:16-33; patch_match_controller.cc:4369-4375, 4706, 4719). */
int smvs_write_maps(smvs_engine* eng, const char* stereo_dir, const char* image_name,
                    const char* output_type);

#ifdef __cplusplus
}
#endif

#endif /* SMVS_H_ */
