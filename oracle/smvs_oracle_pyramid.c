/* smvs_oracle_pyramid.c — CPU oracle of the image pyramid (test infrastructure
 * only; never linked by the product).
 *
 * orc_resample_maps restates ResampleImageBilinear (src/util/mat.cc:18-58),
 * which DepthMap::Rescale and NormalMap::Rescale call through InterpolateImage
 * (mat.cc:129-137; depth_map.cc:32-55, normal_map.cc:27-56), and the normal
 * re-normalisation of NormalMap::Rescale (normal_map.cc:57-72), in the same
 * float expressions. orc_rescale_image restates the separable bilinear
 * (triangle) resampling filter that the reference reaches through FreeImage
 * (Bitmap::Rescale with FILTER_BILINEAR, src/util/bitmap.cc:705-708): the
 * filter half-width is 1 / scale when minifying, weights are normalised over
 * the pixels inside the image, rows first, then columns, and the result is
 * rounded to an integer grey level. FreeImage is a third-party library absent
 * from the reference tree, so this restatement is pinned only against the
 * published algorithm ("parity unpinned" by execution). Compiled with
 * -ffp-contract=off: the CUDA unit performs the same IEEE operations. */
#include <math.h>
#include <stddef.h>

static float pixel_or0(const float* d, int rows, int cols, int r, int c) {
  return (r >= 0 && c >= 0 && r < rows && c < cols) ? d[(size_t)r * cols + c] : 0.0f;
}

int orc_resample_maps(const float* in, int rows, int cols, int planes, int renormalise, float* out, int new_rows,
                      int new_cols) {
  if (!in || !out || rows <= 0 || cols <= 0 || new_rows <= 0 || new_cols <= 0 || planes < 1 || planes > 3) return -1;
  const float scale_r = (float)rows / (float)new_rows;
  const float scale_c = (float)cols / (float)new_cols;
  const size_t in_plane = (size_t)rows * cols, out_plane = (size_t)new_rows * new_cols;
#pragma omp parallel for schedule(static)
  for (int r = 0; r < new_rows; ++r) {
    const float r_i = ((float)r + 0.5f) * scale_r - 0.5f;
    const int r_i_min = (int)floorf(r_i);
    const int r_i_max = r_i_min + 1;
    const float d_r_min = r_i - (float)r_i_min;
    const float d_r_max = (float)r_i_max - r_i;
    for (int c = 0; c < new_cols; ++c) {
      const float c_i = ((float)c + 0.5f) * scale_c - 0.5f;
      const int c_i_min = (int)floorf(c_i);
      const int c_i_max = c_i_min + 1;
      const float d_c_min = c_i - (float)c_i_min;
      const float d_c_max = (float)c_i_max - c_i;
      float v[3];
      for (int p = 0; p < planes; ++p) {
        const float* d = in + p * in_plane;
        const float value1 = d_c_max * pixel_or0(d, rows, cols, r_i_min, c_i_min) +
                             d_c_min * pixel_or0(d, rows, cols, r_i_min, c_i_max);
        const float value2 = d_c_max * pixel_or0(d, rows, cols, r_i_max, c_i_min) +
                             d_c_min * pixel_or0(d, rows, cols, r_i_max, c_i_max);
        v[p] = d_r_max * value1 + d_r_min * value2;
      }
      if (renormalise && planes == 3) {
        const float sq = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        if (sq > 0.f) {
          const float n = sqrtf(sq);
          v[0] = v[0] / n; v[1] = v[1] / n; v[2] = v[2] / n;
        }
      }
      for (int p = 0; p < planes; ++p) out[p * out_plane + (size_t)r * new_cols + c] = v[p];
    }
  }
  return 0;
}

static float filter_at(const float* line, size_t stride, int n, float c, float scale) {
  const float support = scale < 1.0f ? 1.0f / scale : 1.0f;
  const float fscale = scale < 1.0f ? scale : 1.0f;
  int i0 = (int)floorf(c - support), i1 = (int)ceilf(c + support);
  i0 = i0 < 0 ? 0 : i0;
  i1 = i1 > n - 1 ? n - 1 : i1;
  float acc = 0.f, wsum = 0.f;
  for (int i = i0; i <= i1; ++i) {
    const float wt = 1.0f - fabsf(((float)i + 0.5f) - c) * fscale;
    if (wt <= 0.f) continue;
    acc += wt * line[(size_t)i * stride];
    wsum += wt;
  }
  return wsum > 0.f ? acc / wsum : 0.f;
}

int orc_rescale_image(const float* in, int w, int h, float* tmp, float* out, int ow, int oh) {
  if (!in || !tmp || !out || w <= 0 || h <= 0 || ow <= 0 || oh <= 0) return -1;
  const float sx = (float)ow / (float)w, sy = (float)oh / (float)h;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < ow; ++x)
      tmp[(size_t)y * ow + x] = filter_at(in + (size_t)y * w, 1, w, ((float)x + 0.5f) / sx, sx);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < oh; ++y)
    for (int x = 0; x < ow; ++x) {
      const float v = filter_at(tmp + x, (size_t)ow, h, ((float)y + 0.5f) / sy, sy);
      out[(size_t)y * ow + x] = fminf(255.f, fmaxf(0.f, rintf(v)));
    }
  return 0;
}
