/*
 * smvs_testing.h — test hooks of the engine library (not part of the drop-in
 * boundary; no counterpart in the reference).
 */
#ifndef SMVS_TESTING_H_
#define SMVS_TESTING_H_

#include <stddef.h>
#include "smvs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Sample a w*h grey image (values as float, stored on the device in
 * `storage` format: SMVS_STORE_U8 takes round(value) and reads it normalised,
 * F16/F32 store value as is) through the same texture path the cost kernels
 * use (linear filtering, border addressing, unnormalised coordinates) at n
 * coordinates xy[2*i], xy[2*i+1]. Host buffers in and out; synchronous. */
int smvs_test_sample_texture(const float* image, int w, int h, int storage, const float* xy, int n, float* out);

/* Read and clear the CUDA error pending on the calling thread in this
 * library's runtime (cudaGetLastError); returns its code (0 = none). Lets a
 * test start from a clean thread state after other tests. */
int smvs_test_take_cuda_error(void);

/* Benchmark inputs: render one view of the synthetic aerial scene (a terrain
 * of num_hills Gaussian hills {cx, cy, amplitude, sigma} in metres, with
 * num_boxes box buildings {x0, y0, x1, y1, roof height}) by ray casting on the
 * GPU, marching `step` metres along each ray (to at most max_dist metres from
 * the camera, 65536 steps) before bisecting the crossing.
 * K, R, T: intrinsics (3x3 row-major), world-to-camera rotation and
 * translation. Outputs are W*H device buffers: albedo in [0, 1] (seeded value
 * noise with lattice spacing `texel` metres), depth (camera z, 0 where the ray
 * misses) and a planar 3*W*H camera-frame normal facing the camera.
 * Synchronous. */
int smvs_synth_render_aerial(const float* hills, int num_hills, const float* boxes, int num_boxes, uint32_t salt,
                             float texel, float step, float max_dist, const double* K, const double* R,
                             const double* T, int width, int height, float* albedo, float* depth, float* normal,
                             void* stream);

/* Fusion replay waits for the next smvs_fusion_run calls on this thread: each
 * wait for a predecessor gives up after limit_seconds (0 restores the 20 s
 * default) and, if withhold_seed >= 0, that seed never releases its
 * successors (-2: no seed does), so their waits run out and the run returns
 * SMVS_ETIMEDOUT
 * (nothing faults or hangs: every wait is bounded and the kernel finishes). */
int smvs_test_fusion_waits(double limit_seconds, long long withhold_seed);

/* Reference-tile waits of the next smvs_run calls of engine `eng`: each block's
 * wait for its TMA tile gives up after `polls` mbarrier polls (0 restores the
 * default bound), and with skip_copy = 1 the copy is never issued, so every
 * wait runs out; smvs_run's maps are then incomplete and the next
 * smvs_synchronize or getter returns SMVS_ETIMEDOUT. */
int smvs_test_tile_waits(smvs_engine* eng, int polls, int skip_copy);

/* Persistent launches (smvs_tuning.persistent, smvs_pool_options.
 * sweep_persistent) of engines and pools in this process that start a run or
 * build a batch after this call use at most max_blocks blocks (0 restores the
 * resident count), so that small images still have each block loop over many
 * tiles. Maps do not change. */
int smvs_test_persistent_grid(int max_blocks);

/* The propagate-depth initial maps of an engine created with propagate_depth:
 * the given reference maps with the projected source depths composited in
 * (depth W*H, normal 3*W*H planar) and the prior depth (W*H), before random
 * hypotheses fill the pixels still without a depth. Host buffers; synchronous. */
int smvs_test_propagate_init(smvs_engine* eng, float* depth, float* normal, float* prior);

/* The 2-D Delaunay triangulation the Delaunay initial map uses, on n integer
 * points xy[2i], xy[2i + 1] (repeated positions after the first are skipped):
 * *num_tris triangles, their counter-clockwise vertex indices into xy in
 * tris[3k..3k+2] (up to `capacity` triangles written). Host only. */
int smvs_test_delaunay(const int32_t* xy, int n, int32_t* tris, int capacity, int* num_tris);

/* Throughput calibration on the current device, used as roofline denominators
 * for this path's bounds: kind 0 = FP32 FMA rate (flop/s, FMA = 2 flop),
 * kind 1 = bilinear texture samples/s from an 8-bit texture with warp-coherent
 * coordinates (the access pattern of the cost kernels). Runs for about
 * `seconds`; synchronous. */
int smvs_test_calibrate(int kind, double seconds, double* rate);

/* Fusion capacities for the next smvs_fusion_create calls on this thread
 * (0 restores the defaults): records of more than closure_cap pixels go
 * through the overflow closure pass, and records of more than replay_cap
 * pixels or replay_stack stack entries replay from global scratch instead of
 * shared memory. Results do not change; the paths taken do. */
int smvs_test_fusion_caps(int closure_cap, int replay_cap, int replay_stack);

/* With profiling on during smvs_fusion_run: per fused image (in fusion order)
 * the longest chain of seeds that each waited for the previous one (the
 * number of sequential replay steps the image needed) and, optionally, the
 * shear K of its ticket order (key = column + K x row of the seed grid). */
int smvs_test_fusion_chains(smvs_fusion* f, uint32_t* chains, uint32_t* shears, int capacity, int* count);

/* With profiling on: device milliseconds per fused image (in fusion order) and
 * kernel kind (smvs_fusion_kernel), ms[4 * image + kind]. */
int smvs_test_fusion_image_ms(smvs_fusion* f, double* ms, int capacity, int* count);

/* With profiling on: per fused image, the mean microseconds a replayed seed
 * spent waiting for its predecessors and from then until it released its
 * successors, the number of seeds with a record, their mean record size and
 * mean reachable set, how many replayed the traversal one pixel at a time, and
 * the mean microseconds of the three steps after the wait (reading the masks,
 * finding the fused pixels, marking them and releasing): 9 values per image. */
int smvs_test_fusion_replay_times(smvs_fusion* f, double* out, int capacity, int* count);

#ifdef __cplusplus
}
#endif

#endif
