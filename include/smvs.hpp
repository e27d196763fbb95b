// smvs.hpp — header-only C++ RAII wrapper over the C ABI (smvs.h).
//
// Shaped like the reference's operator sensemap::mvs::PatchMatchACMMCuda
// (src/mvs/patch_match_cuda.h:154-203): construct with (options, problem),
// Run() / RunFilter(), then GetDepthMap() / GetNormalMap() / GetConfMap().
// Differences: errors throw smvs::Error (the reference exits the process),
// and maps come back as plain std::vector buffers (W*H, planar slices) that a
// caller converts into its own DepthMap / NormalMap types.
#ifndef SMVS_HPP_
#define SMVS_HPP_

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "smvs.h"

namespace smvs {

struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

inline void Check(int status) {
  if (status != SMVS_OK) throw Error(status, smvs_last_error());
}

inline smvs_options DefaultOptions() {
  smvs_options o;
  Check(smvs_options_default(&o));
  return o;
}

class PatchMatch {
 public:
  PatchMatch(const smvs_options& options, const smvs_problem& problem, void* stream = nullptr) {
    Check(smvs_create(&options, &problem, stream, &eng_));
    Check(smvs_get_size(eng_, &w_, &h_, &n_));
  }
  ~PatchMatch() { smvs_destroy(eng_); }
  PatchMatch(const PatchMatch&) = delete;
  PatchMatch& operator=(const PatchMatch&) = delete;

  bool Run() { Check(smvs_run(eng_)); return true; }
  bool RunFilter(bool deduplication = false) { Check(smvs_run_filter(eng_, deduplication ? 1 : 0)); return true; }

  std::vector<float> GetDepthMap() { return Get<float>(smvs_get_depth_map, (size_t)w_ * h_); }
  std::vector<float> GetNormalMap() { return Get<float>(smvs_get_normal_map, 3 * (size_t)w_ * h_); }
  std::vector<float> GetConfMap() { return Get<float>(smvs_get_conf_map, (size_t)w_ * h_); }
  std::vector<float> GetCostMap() { return Get<float>(smvs_get_cost_map, (size_t)n_ * w_ * h_); }
  std::vector<uint32_t> GetViewSelMap() { return Get<uint32_t>(smvs_get_view_sel_map, (size_t)w_ * h_); }
  std::vector<uint16_t> GetCurvatureMap() { return Get<uint16_t>(smvs_get_curvature_map, 2 * (size_t)w_ * h_); }
  void WriteMaps(const std::string& stereo_dir, const std::string& image_name, const std::string& type) {
    Check(smvs_write_maps(eng_, stereo_dir.c_str(), image_name.c_str(), type.c_str()));
  }

  int width() const { return w_; }
  int height() const { return h_; }
  smvs_engine* handle() { return eng_; }

 private:
  template <typename T, typename Fn>
  std::vector<T> Get(Fn fn, size_t n) {
    std::vector<T> out(n);
    Check(fn(eng_, out.data()));
    return out;
  }
  smvs_engine* eng_ = nullptr;
  int w_ = 0, h_ = 0, n_ = 0;
};

}  // namespace smvs

#endif  // SMVS_HPP_
