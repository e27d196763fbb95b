/*
 * orc_pose.h — the 43-float source pose records of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY, shared by the PatchMatch and cross-filter oracle
 * units. Follows InitTransforms (patch_match_cuda.cu:493-580 for the
 * PatchMatch stage, :1320-1382 for the cross filter) and the pose helpers of
 * src/mvs/utils.cc:14-52, composed in FP64 and rounded to float once.
 */
#ifndef ORC_POSE_H_
#define ORC_POSE_H_

#include "../include/smvs.h"

/* ------------------------------------------------------------------------ */
/* Host pose algebra: utils.cc:14-52 and InitTransforms, patch_match_cuda.cu:493-580 */
/* ------------------------------------------------------------------------ */
static inline void build_poses(const smvs_problem* p, float refK[4], float refiK[4], float* poses) {
  const float* K = p->ref.K;
  refK[0] = K[0]; refK[1] = K[2]; refK[2] = K[4]; refK[3] = K[5];
  refiK[0] = 1.0f / refK[0];
  refiK[1] = -refK[1] / refK[0];
  refiK[2] = 1.0f / refK[2];
  refiK[3] = -refK[3] / refK[2];
  for (int i = 0; i < p->num_src; ++i) {
    const smvs_view* s = &p->src[i];
    double iK[9];
    for (int k = 0; k < 9; ++k) iK[k] = s->K[k];
    const double scale = (s->scale > 0.f) ? s->scale : 1.0;
    if (scale != 1.0) { iK[0] *= scale; iK[2] *= scale; iK[4] *= scale; iK[5] *= scale; }
    double R1[9], T1[3], R2[9], T2[3], R[9], T[3];
    for (int k = 0; k < 9; ++k) { R1[k] = p->ref.R[k]; R2[k] = s->R[k]; }
    for (int k = 0; k < 3; ++k) { T1[k] = p->ref.T[k]; T2[k] = s->T[k]; }
    /* ComputeRelativePose: R = R2 * R1^T, T = T2 - R * T1 (utils.cc:14-26) */
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) {
        double acc = 0;
        for (int k = 0; k < 3; ++k) acc += R2[r * 3 + k] * R1[cc * 3 + k];
        R[r * 3 + cc] = acc;
      }
    for (int r = 0; r < 3; ++r) T[r] = T2[r] - (R[r * 3] * T1[0] + R[r * 3 + 1] * T1[1] + R[r * 3 + 2] * T1[2]);
    /* ComputeProjectionCenter: C = -R^T T (utils.cc:28-33) */
    double C[3];
    for (int r = 0; r < 3; ++r) C[r] = -(R[r] * T[0] + R[3 + r] * T[1] + R[6 + r] * T[2]);
    /* ComposeProjectionMatrix: P = K [R|T] (utils.cc:35-42) */
    double P[12];
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 4; ++cc) {
        double acc = 0;
        for (int k = 0; k < 3; ++k) acc += iK[r * 3 + k] * (cc < 3 ? R[k * 3 + cc] : T[k]);
        P[r * 4 + cc] = acc;
      }
    /* ComposeInverseProjectionMatrix: top rows of [P; 0 0 0 1]^-1 (utils.cc:44-52).
     * Closed form: [R^T K^-1 | -R^T T]. */
    double Ki[9] = {0};
    {
      const double a = iK[0], b = iK[1], cxx = iK[2], d = iK[4], e = iK[5];
      /* K = [a b c; 0 d e; 0 0 1] (iK[3]=iK[6]=iK[7]=0, iK[8]=1 for pinhole K) */
      Ki[0] = 1.0 / a; Ki[1] = -b / (a * d); Ki[2] = (b * e - cxx * d) / (a * d);
      Ki[4] = 1.0 / d; Ki[5] = -e / d; Ki[8] = 1.0;
    }
    double iP[12];
    for (int r = 0; r < 3; ++r) {
      for (int cc = 0; cc < 3; ++cc) {
        double acc = 0;
        for (int k = 0; k < 3; ++k) acc += R[k * 3 + r] * Ki[k * 3 + cc];
        iP[r * 4 + cc] = acc;
      }
      iP[r * 4 + 3] = -(R[r] * T[0] + R[3 + r] * T[1] + R[6 + r] * T[2]);
    }
    float* o = poses + (size_t)i * SMVS_POSE_FLOATS;
    o[0] = (float)iK[0]; o[1] = (float)iK[2]; o[2] = (float)iK[4]; o[3] = (float)iK[5];
    for (int k = 0; k < 9; ++k) o[4 + k] = (float)R[k];
    for (int k = 0; k < 3; ++k) o[13 + k] = (float)T[k];
    for (int k = 0; k < 3; ++k) o[16 + k] = (float)C[k];
    for (int k = 0; k < 12; ++k) o[19 + k] = (float)P[k];
    for (int k = 0; k < 12; ++k) o[31 + k] = (float)iP[k];
  }
}

#endif  /* ORC_POSE_H_ */
