// smvs_io.cpp — SenseMap's on-disk map formats (host only).
//
// Mat<T>::Write/Read (src/util/mat.h:179-215): a text header "W&H&D&" then the
// payload, little endian, slice-major then row-major. NormalMap::Encode/Decode
// (src/mvs/normal_map.cc:137-181): one uint32 per pixel holding two 16-bit
// quantised coordinates. Paths: <stereo>/{depth_maps,normal_maps,conf_maps}/
// <image>.<photometric|geometric>.bin (src/base/common.h:16-33).
#include <cerrno>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "../../include/smvs.h"

namespace {

int SetError(int code, const char* msg, const char* path);

template <typename T>
int WriteMat(const char* path, const T* data, int w, int h, int d) {
  if (!path || !data || w < 0 || h < 0 || d < 0) return SetError(SMVS_EINVAL, "bad arguments to Mat writer", path);
  FILE* f = fopen(path, "wb");
  if (!f) return SetError(SMVS_EIO, "cannot open for writing", path);
  fprintf(f, "%d&%d&%d&", w, h, d);
  const size_t n = (size_t)w * h * d;
  // x86-64 and aarch64 are little endian: the payload is written as is.
  const size_t wrote = fwrite(data, sizeof(T), n, f);
  const int close_rc = fclose(f);
  if (wrote != n || close_rc != 0) return SetError(SMVS_EIO, "short write", path);
  return SMVS_OK;
}

int MkdirP(const std::string& dir) {
  std::string cur;
  for (size_t i = 0; i <= dir.size(); ++i) {
    if (i == dir.size() || dir[i] == '/') {
      if (!cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return -1;
    }
    if (i < dir.size()) cur.push_back(dir[i]);
  }
  return 0;
}

}  // namespace

// smvs_last_error lives in smvs_engine.cu; this translation unit reports
// through the same thread-local slot via a small setter.
extern "C" void smvs_internal_set_error(const char* msg);

namespace {
int SetError(int code, const char* msg, const char* path) {
  std::string m = std::string(msg) + (path ? (std::string(": ") + path) : std::string());
  smvs_internal_set_error(m.c_str());
  return code;
}
}  // namespace

extern "C" {

int smvs_write_mat_f32(const char* path, const float* data, int w, int h, int d) { return WriteMat(path, data, w, h, d); }
int smvs_write_mat_u32(const char* path, const uint32_t* data, int w, int h, int d) { return WriteMat(path, data, w, h, d); }
int smvs_write_mat_u16(const char* path, const uint16_t* data, int w, int h, int d) { return WriteMat(path, data, w, h, d); }

int smvs_read_mat(const char* path, void* data, size_t capacity, int elem_size, int* w, int* h, int* d) {
  if (!path || (elem_size != 2 && elem_size != 4)) return SetError(SMVS_EINVAL, "bad arguments to Mat reader", path);
  FILE* f = fopen(path, "rb");
  if (!f) return SetError(SMVS_EIO, "cannot open for reading", path);
  long ww = 0, hh = 0, dd = 0;
  char c1 = 0, c2 = 0, c3 = 0;
  if (fscanf(f, "%ld%c%ld%c%ld%c", &ww, &c1, &hh, &c2, &dd, &c3) != 6 || c1 != '&' || c2 != '&' || c3 != '&' ||
      ww < 0 || hh < 0 || dd < 0) {
    fclose(f);
    return SetError(SMVS_EIO, "malformed Mat header", path);
  }
  if (w) *w = (int)ww;
  if (h) *h = (int)hh;
  if (d) *d = (int)dd;
  const size_t n = (size_t)ww * hh * dd;
  if (data) {
    if (n * elem_size > capacity) {
      fclose(f);
      return SetError(SMVS_EINVAL, "buffer too small for Mat payload", path);
    }
    if (fread(data, elem_size, n, f) != n) {
      fclose(f);
      return SetError(SMVS_EIO, "truncated Mat payload", path);
    }
  }
  fclose(f);
  return SMVS_OK;
}

// NormalMap::Encode, normal_map.cc:159-181.
int smvs_encode_normal_map(const float* normal, int w, int h, uint32_t* code) {
  if (!normal || !code || w < 0 || h < 0) return SetError(SMVS_EINVAL, "bad arguments to normal encoder", nullptr);
  const float decode_factor = 32767.f;
  const size_t WH = (size_t)w * h;
  for (size_t i = 0; i < WH; ++i) {
    const float n0 = normal[i], n1 = normal[WH + i], n2 = normal[2 * WH + i];
    const float s = (float)((1 - n0) * 0.5);
    const float m = 1.0f / std::sqrt(1 - s);
    float q1 = (float)(n1 * 0.5 * m);
    float q2 = (float)(n2 * 0.5 * m);
    // std::min / std::max as the reference calls them: a NaN (n0 == -1) clamps to +0.999999.
    q1 = std::min(0.999999f, std::max(q1, -0.999999f));
    q2 = std::min(0.999999f, std::max(q2, -0.999999f));
    const uint32_t iq1 = (uint32_t)((q1 + 1) * decode_factor);
    const uint32_t iq2 = (uint32_t)((q2 + 1) * decode_factor);
    code[i] = (iq1 << 16) | iq2;
  }
  return SMVS_OK;
}

// NormalMap::Decode, normal_map.cc:137-157.
int smvs_decode_normal_map(const uint32_t* code, int w, int h, float* normal) {
  if (!normal || !code || w < 0 || h < 0) return SetError(SMVS_EINVAL, "bad arguments to normal decoder", nullptr);
  const float inv = 1.0f / 32767.f;
  const size_t WH = (size_t)w * h;
  for (size_t i = 0; i < WH; ++i) {
    const uint32_t iq1 = code[i] >> 16, iq2 = code[i] & 0x0000ffffu;
    const float q1 = iq1 * inv - 1, q2 = iq2 * inv - 1;
    const float s = q1 * q1 + q2 * q2;
    normal[i] = (float)(1.0 - 2.0 * s);
    normal[WH + i] = (float)(2 * q1 * std::sqrt(1 - s));
    normal[2 * WH + i] = (float)(2 * q2 * std::sqrt(1 - s));
  }
  return SMVS_OK;
}

int smvs_write_maps(smvs_engine* eng, const char* stereo_dir, const char* image_name, const char* output_type) {
  if (!eng || !stereo_dir || !image_name || !output_type)
    return SetError(SMVS_EINVAL, "bad arguments to smvs_write_maps", nullptr);
  int w = 0, h = 0, n = 0;
  int st = smvs_get_size(eng, &w, &h, &n);
  if (st) return st;
  const size_t WH = (size_t)w * h;
  const std::string file = std::string(image_name) + "." + output_type + ".bin";
  const std::string base(stereo_dir);
  std::vector<float> depth(WH), normal(3 * WH), conf(WH);
  if ((st = smvs_get_depth_map(eng, depth.data()))) return st;
  if ((st = smvs_get_normal_map(eng, normal.data()))) return st;
  if ((st = smvs_get_conf_map(eng, conf.data()))) return st;
  std::vector<uint32_t> code(WH);
  smvs_encode_normal_map(normal.data(), w, h, code.data());
  const char* dirs[3] = {"depth_maps", "normal_maps", "conf_maps"};
  for (const char* d : dirs)
    if (MkdirP(base + "/" + d) != 0) return SetError(SMVS_EIO, "cannot create directory", (base + "/" + d).c_str());
  if ((st = smvs_write_mat_f32((base + "/depth_maps/" + file).c_str(), depth.data(), w, h, 1))) return st;
  if ((st = smvs_write_mat_u32((base + "/normal_maps/" + file).c_str(), code.data(), w, h, 1))) return st;
  if ((st = smvs_write_mat_f32((base + "/conf_maps/" + file).c_str(), conf.data(), w, h, 1))) return st;
  return SMVS_OK;
}

}  // extern "C"
