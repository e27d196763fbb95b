// smvs_view_select.cpp — source-view selection and depth ranges from the sparse model.
//
// Host C++ (no device work): Model::GetMaxOverlappingImages (src/mvs/model.cc:
// 701-935), Model::ComputeSharedPoints (:961-999) and Model::ComputeDepthRanges
// (:941-959) with ComputeDepthRangeFromBBox (:23-36), so that a serving loop can
// build PatchMatch problems from a model itself. Images are processed on all
// host threads; results do not depend on the thread count. Where the
// reference's order is unspecified (std::unordered_map iteration followed by an
// unstable sort), ties are broken by image index: equal scores keep ascending
// image order.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <thread>
#include <vector>

#include "../../include/smvs.h"

extern "C" void smvs_internal_set_error(const char* msg);

namespace {

int Fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  smvs_internal_set_error(buf);
  return code;
}

struct V3 {
  double x, y, z;
};
inline V3 Sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double SqNorm(const V3& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline double Norm(const V3& a) { return std::sqrt(SqNorm(a)); }

// ComputeProjectionCenter (src/mvs/utils.cc:28-33): C = -R^T T in float.
V3 Center(const smvs_model_image& im) {
  float c[3];
  for (int r = 0; r < 3; ++r) c[r] = -(im.R[r] * im.T[0] + im.R[3 + r] * im.T[1] + im.R[6 + r] * im.T[2]);
  return {c[0], c[1], c[2]};
}

// CalculateTriangulationAngle (src/base/triangulation.cc:203-224).
double TriangulationAngle(const V3& c1, const V3& c2, const V3& p) {
  const double baseline2 = SqNorm(Sub(c1, c2));
  const double ray1 = SqNorm(Sub(p, c1)), ray2 = SqNorm(Sub(p, c2));
  const double den = 2.0 * std::sqrt(ray1 * ray2);
  if (den == 0.0) return 0.0;
  const double angle = std::abs(std::acos((ray1 + ray2 - baseline2) / den));
  return std::min(angle, M_PI - angle);
}

// Percentile (src/util/math.h:260-275): the element at round(p/100 (n-1)).
float Percentile(std::vector<float> v, double p) {
  const int idx = (int)std::round(p / 100 * (double)(v.size() - 1));
  const size_t k = (size_t)std::max(0, std::min((int)v.size() - 1, idx));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}

template <typename Fn>
void ParallelFor(int n, Fn fn) {
  const int threads = std::max(1, std::min<int>(n, (int)std::thread::hardware_concurrency()));
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (int i; (i = next.fetch_add(1)) < n;) fn(i);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

int smvs_select_views(const smvs_model_image* images, int num_images, const float* points, size_t num_points,
                      const int32_t* track_offsets, const int32_t* track_images, const int32_t* candidates,
                      int num_candidates, int max_num_images, double min_triangulation_angle, int32_t* out_offsets,
                      int32_t* out_images) {
  if (!images || num_images < 1 || (num_points && (!points || !track_offsets || !track_images)) ||
      num_candidates < 0 || (num_candidates && !candidates) || max_num_images < 0 || !out_offsets ||
      (max_num_images && !out_images))
    return Fail(SMVS_EINVAL, "select views: bad arguments");
  const int N = num_images;
  std::vector<char> in_set(N, 0);
  for (int k = 0; k < num_candidates; ++k) {
    if (candidates[k] < 0 || candidates[k] >= N) return Fail(SMVS_EINVAL, "select views: candidate out of range");
    in_set[candidates[k]] = 1;
  }
  if (num_points && track_offsets[0] != 0) return Fail(SMVS_EINVAL, "select views: track_offsets[0] must be 0");
  for (size_t i = 0; i < num_points; ++i) {
    if (track_offsets[i + 1] < track_offsets[i]) return Fail(SMVS_EINVAL, "select views: decreasing track offsets");
    for (int32_t k = track_offsets[i]; k < track_offsets[i + 1]; ++k)
      if (track_images[k] < 0 || track_images[k] >= N) return Fail(SMVS_EINVAL, "select views: track image out of range");
  }
  // Observations per image (:713-720), projection centres (:722-728).
  std::vector<std::vector<uint32_t>> image_points(N);
  for (size_t i = 0; i < num_points; ++i)
    for (int32_t k = track_offsets[i]; k < track_offsets[i + 1]; ++k) image_points[track_images[k]].push_back((uint32_t)i);
  std::vector<V3> C(N);
  for (int i = 0; i < N; ++i) C[i] = Center(images[i]);
  // Shared points (ComputeSharedPoints :961-999) and the mean nearest distance (:731-748).
  std::vector<std::map<int, int>> shared(N);
  for (size_t i = 0; i < num_points; ++i) {
    const int32_t* tr = track_images + track_offsets[i];
    const int t = track_offsets[i + 1] - track_offsets[i];
    for (int a = 0; a < t; ++a)
      for (int b = 0; b < a; ++b)
        if (tr[a] != tr[b]) {
          shared[tr[a]][tr[b]] += 1;
          shared[tr[b]][tr[a]] += 1;
        }
  }
  float m_dist = 0.0f;
  int m_cnt = 0;
  for (int i = 0; i < N; ++i) {
    float md = FLT_MAX;
    for (const auto& s : shared[i]) {
      const float d = (float)Norm(Sub(C[i], C[s.first]));
      if (d <= 1e-5) continue;
      md = std::min(d, md);
    }
    if (md < FLT_MAX) {
      m_dist += md;
      m_cnt++;
    }
  }
  m_dist /= m_cnt;  // 0/0 = NaN when no image shares a point, as in the reference
  const float min_dist = 0.1 * m_dist, max_dist = 100 * m_dist;
  const float min_angle = (float)(0.0 * 0.0174532925199432954743716805978692718781530857086181640625);
  const float max_angle = (float)(60.0 * 0.0174532925199432954743716805978692718781530857086181640625);
  const float min_tri = (float)(min_triangulation_angle * 0.0174532925199432954743716805978692718781530857086181640625);
  std::vector<std::vector<int>> out(N);

  auto select_neighbors = [&](int i1) -> bool {  // :754-822
    const auto& pts = image_points[i1];
    if (pts.empty()) return false;
    std::map<int, int> count;
    std::map<int, std::vector<float>> angles;
    for (uint32_t pi : pts) {
      const V3 X{points[3 * (size_t)pi], points[3 * (size_t)pi + 1], points[3 * (size_t)pi + 2]};
      for (int32_t k = track_offsets[pi]; k < track_offsets[pi + 1]; ++k) {
        const int i2 = track_images[k];
        if (!in_set[i2] || i2 == i1) continue;
        count[i2]++;
        angles[i2].push_back((float)TriangulationAngle(C[i1], C[i2], X));
      }
    }
    const bool rig = images[i1].is_rig != 0;
    std::vector<std::pair<int, int>> ordered;
    for (const auto& c : count)
      if (Percentile(angles[c.first], 75) >= min_tri) {
        const double factor = (images[c.first].is_rig != 0) == rig ? 1.5 : 1.0;
        ordered.emplace_back(c.first, (int)(c.second * factor));
      }
    std::stable_sort(ordered.begin(), ordered.end(),
                     [](const std::pair<int, int>& a, const std::pair<int, int>& b) { return a.second > b.second; });
    const size_t eff = std::min(ordered.size(), (size_t)max_num_images);
    for (size_t k = 0; k < eff; ++k) out[i1].push_back(ordered[k].first);
    return true;
  };

  auto select_spatial = [&](int i1) {  // :823-905
    const float* R1 = images[i1].R;
    const float ref_ray[3] = {R1[6], R1[7], R1[8]};
    struct Score {
      int idx;
      float score;
    };
    std::vector<Score> scores;
    for (int i = 0; i < N; ++i) {
      if (i == i1) continue;
      const float* R2 = images[i].R;
      const float src_ray[3] = {R2[6], R2[7], R2[8]};
      const float dist = (float)Norm(Sub(C[i], C[i1]));
      if (dist < min_dist || dist > max_dist) continue;
      const float cos_angle = ref_ray[0] * src_ray[0] + ref_ray[1] * src_ray[1] + ref_ray[2] * src_ray[2];
      const float angle = std::acos(cos_angle);
      if (angle < min_angle || angle > max_angle) continue;
      const float wangle = 1.1f - cos_angle;
      const float wdist = std::max(dist / m_dist, 1.0f);
      scores.push_back({i, wangle * wdist});
    }
    std::stable_sort(scores.begin(), scores.end(), [](const Score& a, const Score& b) { return a.score < b.score; });
    const size_t eff = std::min(scores.size(), (size_t)max_num_images);
    if (eff < 1) return;
    std::vector<int> sel{i1};
    while (sel.size() <= eff && !scores.empty()) {
      size_t k;
      for (k = 0; k < scores.size(); ++k) {
        const int next = scores[k].idx;
        bool spurious = false;
        for (int o : sel)
          if (Norm(Sub(C[next], C[o])) < min_dist) {
            spurious = true;
            break;
          }
        if (!spurious) {
          sel.push_back(next);
          scores.erase(scores.begin() + k);
          break;
        }
      }
      if (k >= scores.size()) break;
    }
    out[i1].assign(sel.begin() + 1, sel.end());
  };

  std::vector<int> todo;
  for (int i = 0; i < N; ++i)
    if (in_set[i]) todo.push_back(i);
  ParallelFor((int)todo.size(), [&](int k) {
    if (!select_neighbors(todo[k])) select_spatial(todo[k]);
  });
  out_offsets[0] = 0;
  for (int i = 0; i < N; ++i) {
    for (size_t k = 0; k < out[i].size(); ++k) out_images[(size_t)out_offsets[i] + k] = out[i][k];
    out_offsets[i + 1] = out_offsets[i] + (int32_t)out[i].size();
  }
  return SMVS_OK;
}

int smvs_compute_depth_ranges(const smvs_model_image* images, int num_images, const float bbox_lt[3],
                              const float bbox_rb[3], float* ranges) {
  if (!images || num_images < 0 || !bbox_lt || !bbox_rb || (num_images && !ranges))
    return Fail(SMVS_EINVAL, "depth ranges: bad arguments");
  // BoundingBox::GetCorners (src/util/bb.h:86-96).
  const float* lt = bbox_lt;
  const float* rb = bbox_rb;
  const float corners[8][3] = {{lt[0], lt[1], lt[2]}, {rb[0], lt[1], lt[2]}, {rb[0], rb[1], lt[2]},
                               {lt[0], rb[1], lt[2]}, {lt[0], lt[1], rb[2]}, {rb[0], lt[1], rb[2]},
                               {rb[0], rb[1], rb[2]}, {lt[0], rb[1], rb[2]}};
  for (int i = 0; i < num_images; ++i) {
    const float* R = images[i].R;
    const float* t = images[i].T;
    float lo = 0, hi = 0;
    for (int k = 0; k < 8; ++k) {
      const float z = R[6] * corners[k][0] + R[7] * corners[k][1] + R[8] * corners[k][2] + t[2];
      lo = k ? std::min(lo, z) : z;
      hi = k ? std::max(hi, z) : z;
    }
    ranges[2 * i] = std::max(0.000001f, lo);
    ranges[2 * i + 1] = hi;
  }
  return SMVS_OK;
}

}  // extern "C"
