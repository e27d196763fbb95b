/*
 * smvs_oracle.h — CPU oracle for the PatchMatch depth-map path.
 *
 * TEST INFRASTRUCTURE ONLY. This is an OpenMP transcription of the reference
 * kernel logic (SenseMap src/mvs/kernel_functions.cu, patch_match_cuda.cu,
 * gpu_mat_ref_image.cu, utils.{h,cc}), labelled as such: the reference has no
 * CPU PatchMatch of its own. It is the checker for the CUDA engine in
 * sensemap_b200/csrc and the timed CPU baseline of bench.py; the product never
 * links or calls it.
 *
 * Deliberate differences from the reference, each shared with the CUDA engine:
 *   - cuRAND XORWOW is replaced by a counter-based generator (splitmix64 mixing,
 *     Steele, Lea & Flood, OOPSLA 2014) keyed on (seed, stage, pixel, draw);
 *   - the Marsaglia normal sampler gives up after 32 rejected trials.
 * Parity against the reference's own kernels is checked by running them (built
 * from the reference sources into oracle/_ref by oracle/ref_build.py) on the
 * same inputs: cost-level parity deterministically, full runs statistically.
 */
#ifndef SMVS_ORACLE_H_
#define SMVS_ORACLE_H_

#include <stdint.h>
#include "../include/smvs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Outputs of one oracle run (caller-owned, dense). Any pointer may be NULL. */
typedef struct orc_outputs {
  float* depth;      /* W*H */
  float* normal;     /* 3*W*H planar */
  float* conf;       /* W*H */
  float* cost;       /* N*W*H planar */
  uint32_t* view_sel;/* W*H */
  float* grad;       /* W*H  (ComputeGradientMap) */
  float* ref_sum;    /* W*H  (bilateral mean of the reference window) */
  float* ref_sqsum;  /* W*H  (bilateral mean of squares) */
  float* poses;      /* N*43 */
  uint16_t* curvature; /* 2*W*H (est_curvature && geom_consistency) */
} orc_outputs;

/* PatchMatchACMMCuda(options, problem) + Run() on the CPU, rows [row_begin,
 * row_end) of every half-sweep only when row_end > row_begin (a bounded band
 * used for CPU timing), else the whole image. Host memory only. */
int orc_run(const smvs_options* opt, const smvs_problem* prob, int row_begin, int row_end,
            orc_outputs* out);

/* The propagate-depth initial maps (InitWorkspace, patch_match_cuda.cu:603-659):
 * every source with a depth map (src[i].depth) is projected into the W x H
 * reference view with its pose record (poses: N*43), pixels of `depth` that
 * are <= 0 take the median (or the first / smaller of two) projected depth,
 * `prior` (W*H) receives the medians that more than two projections agree
 * with, and `normal` (3*W*H planar) is fitted to the result. depth and normal
 * hold the given maps on entry. */
int orc_propagate_init(int W, int H, int N, const float refK[4], const float refiK[4], const float* poses,
                       const smvs_view* src, float* depth, float* normal, float* prior);
/* The same for a PatchMatch problem (host memory): its pose records, with the
 * given maps ref.depth / ref.normal copied into depth / normal first. */
int orc_propagate_init_problem(const smvs_problem* prob, float* depth, float* normal, float* prior);

/* PatchMatchACMMCuda::RunFilter(false): FilterDepthMapsKernel over the
 * problem's ref.depth using the source views' depth maps. Writes W*H. */
int orc_run_filter(const smvs_options* opt, const smvs_problem* prob, float* depth_out);

/* Cost of one hypothesis at sampled pixels, FP32 transcription (same as the
 * run) and FP64 evaluation (bilinear in double, exact exp/sqrt, unquantised
 * texture weights). costs32/costs64 are n_pix*N. */
int orc_eval_costs(const smvs_options* opt, const smvs_problem* prob, int n_pix,
                   const int* rows, const int* cols, const float* depths,
                   const float* normals /* n_pix*3 */, float* costs32, double* costs64);

/* CrossFilterCuda::Run over a view set (patch_match_cuda.cu:1493-1559): for each
 * problem with at least one source, refined[ref] (W*H of the reference view) is
 * written; other entries of `refined` are not touched and may be NULL. */
int orc_cross_filter_run(const smvs_options* opt, const smvs_filter_view* views, int num_views,
                         const smvs_filter_problem* problems, int num_problems, float* const* refined);

/* CrossFilterCuda::DedupRun (:1561-1625). Dedup input of view v: refined[v]
 * when views[v].ref_flag (an all-zero map when refined or refined[v] is NULL),
 * else views[v].depth. vis[v] (W*H, every view) is initialised and updated;
 * delta[ref] (W*H) is written for each problem with at least one source. */
int orc_cross_filter_dedup(const smvs_options* opt, const smvs_filter_view* views, int num_views,
                           const smvs_filter_problem* problems, int num_problems, const float* const* refined,
                           uint32_t* const* vis, float* const* delta);

/* GetDeduplicDepthMap (:1641-1664) of one view after orc_cross_filter_dedup. */
int orc_cross_filter_dedup_depth(const smvs_filter_view* view, const float* refined, const uint32_t* vis,
                                 float* out);

/* The reference K, its inverse and the 43-float source pose records of one
 * cross-filter problem (InitTransforms, patch_match_cuda.cu:1320-1407). */
int orc_cross_filter_poses(const smvs_filter_view* views, int num_views, const smvs_filter_problem* problem,
                           float refK[4], float refiK[4], float* poses);

/* NormalMap::Encode (normal_map.cc:159-181) of a planar 3*W*H map. */
int orc_encode_normal_map(const float* normal, int width, int height, uint32_t* code);

/* Initial maps from the model (patch_match_controller.cc): InitDepthMap +
 * InitDepthMapFromSparsePoint (:1205-1307, :483-518), Model2Depth (:520-642),
 * Ply2Depth (:643-750). `view` gives width, height, K, R, T; depth is W*H,
 * normal 3*W*H planar; range[2] is the returned depth range. */
/* Delaunay initial map (InitDepthMapFromDelaunay, :398-474): the projected
 * points that land in the view (input order; uv 2 per point, z, input index),
 * and the map rasterised from a triangulation of them (counter-clockwise
 * index triples into that list). */
int orc_delaunay_points(const smvs_view* v, const float* xyz, size_t n, int32_t* uv, float* z, int32_t* idx,
                        size_t* count);
int orc_init_from_delaunay(const smvs_view* v, const float* xyz, size_t n, const int32_t* tris, size_t ntri,
                           float* depth, float* normal, float* range);
int orc_init_from_sparse_points(const smvs_view* view, const float* xyz, size_t n, float* depth, float* normal,
                                float* range);
int orc_init_from_mesh(const smvs_view* view, const double* vertices, size_t num_vertices, const int32_t* faces,
                       size_t num_faces, const double* face_normals, float* depth, float* normal, float* range);
int orc_init_from_dense_points(const smvs_view* view, const float* xyz, const float* normals, size_t n, int level,
                               float* depth, float* normal, float* range);

/* ---- fusion (smvs_oracle_fusion.c) ---- */
/* StereoFusion::Run for one cluster of every image; max_images > 0 stops after
 * that many images. Returns a result handle, NULL on bad arguments or no memory. */
void* orc_fusion_run(const smvs_fusion_options* opt, const smvs_fusion_view* views, int num_views,
                     const int32_t* overlap_offsets, const int32_t* overlap_images, int max_images);
/* The same with the reference's concurrent row slices on `threads` threads
 * (threads > 1): a timing baseline whose results depend on the timing. */
void* orc_fusion_run_threads(const smvs_fusion_options* opt, const smvs_fusion_view* views, int num_views,
                             const int32_t* overlap_offsets, const int32_t* overlap_images, int max_images,
                             int threads);
int orc_fusion_sizes(void* h, size_t* num_points, size_t* num_vis, int* order_count);
int orc_fusion_copy(void* h, smvs_fused_point* points, uint64_t* vis_offsets, uint32_t* vis_images, int* order);
int orc_fusion_mask(void* h, int view, int width, int height, uint8_t* out);
void orc_fusion_free(void* h);

/* RemoveDuplicatePoints (fusion.cc:2184-2266) over a fused cloud: keep[i] = 0
 * for the points it drops. */
int orc_fusion_duplicate_keep(const smvs_fusion_view* views, int nv, const smvs_fused_point* pts, size_t n,
                              const uint64_t* off, const uint32_t* vis, uint8_t* keep);
/* RemoveOutliers (fusion.cc:2542-2611) with ComputeAverageDistance
 * (patch_match_controller.cc:115-228) by brute-force neighbours: scores[n]
 * updated in place, keep[n], spacing[n] (may be NULL). */
int orc_fusion_outlier_keep(const smvs_fused_point* pts, size_t n, int nb, double max_spacing_factor, float* scores,
                            uint8_t* keep, float* spacing);

/* The generator shared with the engine: uniform in (0, 1]. */
float orc_uniform(uint64_t seed, uint32_t stage, uint32_t pixel, uint32_t draw);

/* Texture filtering model used by the oracle (CUDA linear filtering with
 * 8-bit fixed-point weights): sample `img` (w*h floats) at unnormalised (x, y). */
float orc_tex_bilinear(const float* img, int w, int h, float x, float y);

/* Number of OpenMP threads the oracle uses. */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif
