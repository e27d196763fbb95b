// smvs_device.cuh — device-side building blocks of the PatchMatch engine.
//
// Each helper restates one device function of the reference
// (src/mvs/kernel_functions.cu, src/mvs/utils.h) for sm_100a; the citations
// give the file:line it follows. Reference quirks that change results are
// kept and marked "[quirk]" so that outputs match the reference's.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/smvs.h"

namespace smvs {

constexpr int kMaxHyp = 11;  // K_NUM_SAMPS + 3 (kernel_functions.h:32)
constexpr int kMarsagliaTrials = 32;
constexpr uint32_t kStageInit = 1u;

__host__ __device__ inline uint32_t StageSweep(int iter, int colour) { return 2u + 4u * iter + colour; }
__host__ __device__ inline uint32_t StageLocal(int iter, int colour) { return 4u + 4u * iter + colour; }

// ---------------------------------------------------------------------------
// Counter-based RNG replacing cuRAND XORWOW (gpu_mat_prng.cu:10-37): draws are
// a pure function of (seed, stage, pixel, draw index), mixed with the
// splitmix64 finaliser (Steele, Lea & Flood, OOPSLA 2014). No state array.
// ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t Mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t StageKey(uint64_t seed, uint32_t stage) {
  return Mix64(seed + 0x632BE59BD9B4E019ULL * (uint64_t)(stage + 1u));
}
struct Rng {
  uint64_t key;
  uint32_t draw;
  __device__ Rng(uint64_t stage_key, uint32_t pixel) : key(Mix64(stage_key + (uint64_t)pixel)), draw(0) {}
  // Uniform in (0, 1], like curand_uniform.
  __device__ float Uniform() {
    const uint64_t x = Mix64(key + 0x9E3779B97F4A7C15ULL * (uint64_t)(draw + 1u));
    ++draw;
    return (float)((x >> 40) + 1u) * (1.0f / 16777216.0f);
  }
};

__device__ __forceinline__ float Dot3(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// GenerateRandomNormal (view-ray form), kernel_functions.cu:112-139; Marsaglia's
// sphere sampler, bounded to kMarsagliaTrials rejections.
__device__ inline void RandomNormal(Rng& r, const float view_ray[3], float n[3]) {
  float v1 = 0.f, v2 = 0.f, s = 2.0f;
  for (int t = 0; t < kMarsagliaTrials && s >= 1.0f; ++t) {
    v1 = 2.0f * r.Uniform() - 1.0f;
    v2 = 2.0f * r.Uniform() - 1.0f;
    s = v1 * v1 + v2 * v2;
  }
  if (s >= 1.0f) {
    n[0] = 0.f; n[1] = 0.f; n[2] = -1.0f;
    return;
  }
  const float s_norm = 2.0f * sqrtf(1.0f - s);
  n[0] = v1 * s_norm;
  n[1] = v2 * s_norm;
  n[2] = 1.0f - 2.0f * s;
  if (Dot3(n, view_ray) > 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
}

// CorrectNormal, kernel_functions.cu:227-306.
__device__ inline void CorrectNormal(float n[3], const float vd[3], float inv_view_len) {
  const float cal = Dot3(n, vd);
  if (cal >= 0) {
    float c3[3];
    c3[0] = n[1] * vd[2] - n[2] * vd[1];
    c3[1] = n[2] * vd[0] - n[0] * vd[2];
    c3[2] = n[0] * vd[1] - n[1] * vd[0];
    float phi = (float)((double)acosf(cal * inv_view_len) - 90.0 * 0.0174532925199432);
    phi = fminf(phi * 1.01f, -0.001f);
    if (phi == 0) return;
    const float icl = rsqrtf(c3[0] * c3[0] + c3[1] * c3[1] + c3[2] * c3[2]);
    c3[0] *= icl; c3[1] *= icl; c3[2] *= icl;
    const float om[9] = {0.0f, -c3[2], c3[1], c3[2], 0.0f, -c3[0], -c3[1], c3[0], 0.0f};
    const float sp = __sinf(phi);
    const float cp = 1.0f - __cosf(phi);
    float cO[9];
    cO[0] = cp * (om[0] * om[0] + om[1] * om[3] + om[2] * om[6]);
    cO[1] = cp * (om[0] * om[1] + om[1] * om[4] + om[2] * om[7]);
    cO[2] = cp * (om[0] * om[2] + om[1] * om[5] + om[2] * om[8]);
    cO[3] = cp * (om[3] * om[0] + om[4] * om[3] + om[5] * om[6]);
    cO[4] = cO[3];  // [quirk] :272-276 copy entries instead of computing them
    cO[5] = cO[3];
    cO[6] = cp * (om[6] * om[0] + om[7] * om[3] + om[8] * om[6]);
    cO[7] = cO[6];
    cO[8] = cO[6];
    float Rt[9];
    Rt[0] = 1 + om[0] * sp + cO[0]; Rt[1] = 0 + om[1] * sp + cO[1]; Rt[2] = 0 + om[2] * sp + cO[2];
    Rt[3] = 0 + om[3] * sp + cO[3]; Rt[4] = 1 + om[4] * sp + cO[4]; Rt[5] = 0 + om[5] * sp + cO[5];
    Rt[6] = 0 + om[6] * sp + cO[6]; Rt[7] = 0 + om[7] * sp + cO[7]; Rt[8] = 1 + om[8] * sp + cO[8];
    const float r0 = Rt[0] * n[0] + Rt[1] * n[1] + Rt[2] * n[2];
    const float r1 = Rt[3] * n[0] + Rt[4] * n[1] + Rt[5] * n[2];
    const float r2 = Rt[6] * n[0] + Rt[7] * n[1] + Rt[8] * n[2];
    n[0] = r0; n[1] = r1; n[2] = r2;
  }
}

// PropagateDepth (normalised-point form), kernel_functions.cu:409-429.
__device__ __forceinline__ float PropagateDepth(float d1, const float n1[3], const float iK[4], int row1,
                                                int col1, const float p2[3]) {
  const float x1 = d1 * (iK[0] * col1 + iK[1]);
  const float y1 = d1 * (iK[2] * row1 + iK[3]);
  const float d = n1[0] * x1 + n1[1] * y1 + n1[2] * d1;
  const float t = d / (n1[0] * p2[0] + n1[1] * p2[1] + n1[2] * p2[2]);
  if (fabsf(t) < 1e-5f) return d1;
  return t;
}

// PerturbNormal (ACMH form) via Normal2Dir / Dir2Normal: kernel_functions.cu:214-225,
// utils.h:94-106.
__device__ __forceinline__ void PerturbNormalACMH(const float n[3], float out[3], float a1, float a2, Rng& r) {
  const float y = atan2f(sqrtf(n[0] * n[0] + n[1] * n[1]), n[2]);
  const float x = atan2f(n[1], n[0]);
  const float nx = a1 * (2 * r.Uniform() - 1) + x;
  const float ny = a2 * (2 * r.Uniform() - 1) + y;
  const float sy = __sinf(ny);
  out[0] = __cosf(nx) * sy;
  out[1] = __sinf(nx) * sy;
  out[2] = __cosf(ny);
}

// ComposeHomography, kernel_functions.cu:431-503. H maps reference pixel
// (col, row, 1) to the source view for the plane (depth, n).
__device__ __forceinline__ void ComposeHomography(const float* pose, int row, int col, float depth,
                                                  const float n[3], const float iK[4], float H[9]) {
  const float* K = pose;
  const float* R = pose + 4;
  const float* T = pose + 13;
  const float dist = depth * (n[0] * (iK[0] * col + iK[1]) + n[1] * (iK[2] * row + iK[3]) + n[2]);
  const float inv_dist = 1.0f / dist;
  const float N0 = inv_dist * n[0], N1 = inv_dist * n[1], N2 = inv_dist * n[2];
  const float K0R0N0T0 = K[0] * (R[0] + N0 * T[0]);
  const float K0R1N1T0 = K[0] * (R[1] + N1 * T[0]);
  const float K2R3N0T1 = K[2] * (R[3] + N0 * T[1]);
  const float K2R4N1T1 = K[2] * (R[4] + N1 * T[1]);
  const float R6N0T2 = R[6] + N0 * T[2];
  const float R7N1T2 = R[7] + N1 * T[2];
  const float A = K0R0N0T0 + K[1] * R6N0T2;
  const float B = K0R1N1T0 + K[1] * R7N1T2;
  const float C = K2R3N0T1 + K[3] * R6N0T2;
  const float D = K2R4N1T1 + K[3] * R7N1T2;
  const float R8 = R[8] + N2 * T[2];
  H[0] = iK[0] * A;
  H[1] = iK[2] * B;
  H[2] = K[0] * (R[2] + N2 * T[0]) + K[1] * R8 + iK[1] * A + iK[3] * B;
  H[3] = iK[0] * C;
  H[4] = iK[2] * D;
  H[5] = K[2] * (R[5] + N2 * T[1]) + K[3] * R8 + iK[1] * C + iK[3] * D;
  H[6] = iK[0] * R6N0T2;
  H[7] = iK[2] * R7N1T2;
  H[8] = iK[1] * R6N0T2 + iK[3] * R7N1T2 + R8;
}

// ComputeGeomConsistencyCostShared, kernel_functions.cu:505-568: forward project,
// bilinear source depth (texture, border 0), back-project, reproject.
__device__ __forceinline__ float GeomCost(const float* pose, cudaTextureObject_t dep_tex, float row, float col,
                                          float depth, const float np[3], const float K[4], float max_cost) {
  const float* P = pose + 19;
  const float* iP = pose + 31;
  const float X0 = depth * np[0], X1 = depth * np[1], X2 = depth * np[2];
  const float ifz = 1.0f / (P[8] * X0 + P[9] * X1 + P[10] * X2 + P[11]);
  float scol = ifz * (P[0] * X0 + P[1] * X1 + P[2] * X2 + P[3]);
  float srow = ifz * (P[4] * X0 + P[5] * X1 + P[6] * X2 + P[7]);
  const float sd = tex2D<float>(dep_tex, scol + 0.5f, srow + 0.5f);
  if (sd == 0.0f) return max_cost;
  scol *= sd;
  srow *= sd;
  const float bx = iP[0] * scol + iP[1] * srow + iP[2] * sd + iP[3];
  const float by = iP[4] * scol + iP[5] * srow + iP[6] * sd + iP[7];
  const float bz = iP[8] * scol + iP[9] * srow + iP[10] * sd + iP[11];
  const float ibz = 1.0f / bz;
  const float bcol = ibz * K[0] * bx + K[1];
  const float brow = ibz * K[2] * by + K[3];
  const float dc = col - bcol, dr = row - brow;
  return fminf(max_cost, sqrtf(dc * dc + dr * dr));
}

}  // namespace smvs
