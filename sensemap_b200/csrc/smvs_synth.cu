// smvs_synth.cu — ray-caster of the synthetic aerial scene (benchmark inputs).
//
// The benchmark's aerial configurations need hundreds of large views of a
// terrain heightfield with box buildings, with analytic ground-truth depth and
// normals. This unit renders one view per call on the GPU: every pixel's ray
// (camera-z = 1 parameterisation, so the ray parameter is the depth) marches
// through the slab of surface heights in fixed world-length steps, then bisects
// the crossing. The surface is a 2.5-D heightfield: the terrain (a sum of
// Gaussian hills) or, inside a building's footprint, the building's roof when
// that is higher. Buildings are found through a uniform grid of cells (CSR
// lists of the boxes that overlap each cell). The albedo is seeded value noise
// (three octaves) on the ground and roofs, and on the wall plane for walls.
// Results are compute only, independent of any graphics API.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/smvs.h"

extern "C" void smvs_internal_set_error(const char* msg);

namespace {

constexpr int kMaxHills = 64;

struct SynthScene {
  int num_hills;
  float hills[kMaxHills][4];  // cx, cy, amplitude, sigma (metres)
  float z_lo, z_hi;           // slab holding every surface point
  float grid_x0, grid_y0, cell;
  int grid_nx, grid_ny;
  const int* cell_start;      // grid_nx * grid_ny + 1
  const int* cell_boxes;      // box indices
  const float* boxes;         // x0, y0, x1, y1, top (5 floats per box)
  uint32_t salt;
};

struct SynthCamera {
  float C[3];     // centre
  float Rt[9];    // camera-to-world rotation (R transposed)
  float iK[4];    // 1/fx, -cx/fx, 1/fy, -cy/fy
  float R[9];     // world-to-camera rotation
  int W, H;
};

__device__ __forceinline__ float Terrain(const SynthScene& s, float x, float y, float* gx, float* gy) {
  float h = 0.f, hx = 0.f, hy = 0.f;
  for (int i = 0; i < s.num_hills; ++i) {
    const float dx = x - s.hills[i][0], dy = y - s.hills[i][1];
    const float is2 = 1.0f / (s.hills[i][3] * s.hills[i][3]);
    const float e = s.hills[i][2] * __expf(-0.5f * (dx * dx + dy * dy) * is2);
    h += e;
    hx -= e * dx * is2;
    hy -= e * dy * is2;
  }
  if (gx) { *gx = hx; *gy = hy; }
  return h;
}

// Highest roof whose footprint holds (x, y), or -inf; *box gets its index.
__device__ __forceinline__ float Roof(const SynthScene& s, float x, float y, int* box) {
  const int cx = (int)floorf((x - s.grid_x0) / s.cell), cy = (int)floorf((y - s.grid_y0) / s.cell);
  float top = -INFINITY;
  *box = -1;
  if (cx < 0 || cy < 0 || cx >= s.grid_nx || cy >= s.grid_ny) return top;
  const int c = cy * s.grid_nx + cx;
  for (int k = s.cell_start[c]; k < s.cell_start[c + 1]; ++k) {
    const int b = s.cell_boxes[k];
    const float* B = s.boxes + 5 * b;
    if (x >= B[0] && x <= B[2] && y >= B[1] && y <= B[3] && B[4] > top) { top = B[4]; *box = b; }
  }
  return top;
}

__device__ __forceinline__ float Height(const SynthScene& s, float x, float y) {
  int box;
  return fmaxf(Terrain(s, x, y, nullptr, nullptr), Roof(s, x, y, &box));
}

__device__ __forceinline__ uint32_t Hash(int ix, int iy, uint32_t salt) {
  uint32_t h = (uint32_t)ix * 0x8da6b343u ^ (uint32_t)iy * 0xd8163841u ^ salt * 0xcb1ab31fu;
  h ^= h >> 13;
  h *= 0x5bd1e995u;
  h ^= h >> 15;
  return h;
}

// Value noise in [0, 1): three octaves of smoothstep-interpolated lattice values.
__device__ float ValueNoise(float u, float v, uint32_t salt) {
  float total = 0.f, amp = 1.f, norm = 0.f;
  for (int o = 0; o < 3; ++o) {
    const float fu = floorf(u), fv = floorf(v);
    const int iu = (int)fu, iv = (int)fv;
    float a = u - fu, b = v - fv;
    a = a * a * (3.f - 2.f * a);
    b = b * b * (3.f - 2.f * b);
    const float v00 = (Hash(iu, iv, salt + o) >> 8) * (1.0f / 16777216.0f);
    const float v10 = (Hash(iu + 1, iv, salt + o) >> 8) * (1.0f / 16777216.0f);
    const float v01 = (Hash(iu, iv + 1, salt + o) >> 8) * (1.0f / 16777216.0f);
    const float v11 = (Hash(iu + 1, iv + 1, salt + o) >> 8) * (1.0f / 16777216.0f);
    total += amp * ((v00 * (1 - a) + v10 * a) * (1 - b) + (v01 * (1 - a) + v11 * a) * b);
    norm += amp;
    amp *= 0.5f;
    u *= 2.03f;
    v *= 2.03f;
  }
  return total / norm;
}

// Rays end at max_dist metres from the camera (and after at most kMaxSteps
// steps): farther surfaces are left empty (depth 0).
constexpr int kMaxSteps = 1 << 16;

__global__ void RenderAerialKernel(SynthScene s, SynthCamera cam, float texel, float step, float max_dist,
                                   float* __restrict__ albedo, float* __restrict__ depth, float* __restrict__ normal) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= cam.W || row >= cam.H) return;
  const size_t pix = (size_t)row * cam.W + col;
  const size_t WH = (size_t)cam.W * cam.H;
  const float pc[3] = {cam.iK[0] * col + cam.iK[1], cam.iK[2] * row + cam.iK[3], 1.0f};
  float d[3];
  for (int i = 0; i < 3; ++i) d[i] = cam.Rt[3 * i] * pc[0] + cam.Rt[3 * i + 1] * pc[1] + cam.Rt[3 * i + 2];
  albedo[pix] = 0.f;
  depth[pix] = 0.f;
  normal[pix] = 0.f; normal[WH + pix] = 0.f; normal[2 * WH + pix] = 0.f;
  if (!(d[2] < -1e-6f)) return;  // the ray never descends to the surface
  const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const float t_in = fmaxf(0.f, (s.z_hi - cam.C[2]) / d[2]);
  const float t_out = fminf((s.z_lo - cam.C[2]) / d[2], max_dist / len);
  if (t_in > t_out) return;
  const float dt = fmaxf(step / len, (t_out - t_in) / (float)kMaxSteps);
  float t_prev = t_in, t_hit = -1.f;
  for (int k = 0; k <= kMaxSteps + 1; ++k) {
    const float t = t_in + k * dt;
    if (t > t_out + dt) break;
    const float x = cam.C[0] + t * d[0], y = cam.C[1] + t * d[1], z = cam.C[2] + t * d[2];
    if (z <= Height(s, x, y)) { t_hit = t; break; }
    t_prev = t;
  }
  if (t_hit < 0.f) return;
  float lo = t_prev, hi = t_hit;
  for (int i = 0; i < 32; ++i) {
    const float mid = 0.5f * (lo + hi);
    const float x = cam.C[0] + mid * d[0], y = cam.C[1] + mid * d[1], z = cam.C[2] + mid * d[2];
    if (z <= Height(s, x, y)) hi = mid; else lo = mid;
  }
  const float t = 0.5f * (lo + hi);
  const float x = cam.C[0] + t * d[0], y = cam.C[1] + t * d[1], z = cam.C[2] + t * d[2];
  // Classify the hit: roof, wall (the ray entered a footprint between lo and hi
  // below its roof), or terrain.
  float gx, gy;
  const float ht = Terrain(s, x, y, &gx, &gy);
  int box_in;
  const float roof_hi = Roof(s, cam.C[0] + hi * d[0], cam.C[1] + hi * d[1], &box_in);
  float n[3];
  float a;
  const float texscale = 1.0f / texel;
  if (box_in >= 0 && roof_hi > ht && z < roof_hi - 1e-3f) {
    // Wall: outward normal of the footprint face crossed.
    const float* B = s.boxes + 5 * box_in;
    const float xl = cam.C[0] + lo * d[0], yl = cam.C[1] + lo * d[1];
    n[0] = 0.f; n[1] = 0.f; n[2] = 0.f;
    float along;
    if (xl < B[0]) { n[0] = -1.f; along = y; }
    else if (xl > B[2]) { n[0] = 1.f; along = y; }
    else if (yl < B[1]) { n[1] = -1.f; along = x; }
    else { n[1] = 1.f; along = x; }
    a = ValueNoise(along * texscale, z * texscale, s.salt ^ 0x51ed27u);
  } else if (box_in >= 0 && roof_hi > ht) {
    n[0] = 0.f; n[1] = 0.f; n[2] = 1.f;
    a = ValueNoise(x * texscale, y * texscale, s.salt ^ 0x2f9bu);
  } else {
    const float inv = rsqrtf(gx * gx + gy * gy + 1.f);
    n[0] = -gx * inv; n[1] = -gy * inv; n[2] = inv;
    a = ValueNoise(x * texscale, y * texscale, s.salt);
  }
  // Normal in the camera frame, facing the camera.
  float nc[3];
  for (int i = 0; i < 3; ++i) nc[i] = cam.R[3 * i] * n[0] + cam.R[3 * i + 1] * n[1] + cam.R[3 * i + 2] * n[2];
  if (nc[0] * pc[0] + nc[1] * pc[1] + nc[2] * pc[2] > 0.f) { nc[0] = -nc[0]; nc[1] = -nc[1]; nc[2] = -nc[2]; }
  albedo[pix] = 0.12f + 0.76f * a;
  depth[pix] = t;
  normal[pix] = nc[0]; normal[WH + pix] = nc[1]; normal[2 * WH + pix] = nc[2];
}

int Fail(int code, const char* msg) {
  smvs_internal_set_error(msg);
  return code;
}

}  // namespace

extern "C" int smvs_synth_render_aerial(const float* hills, int num_hills, const float* boxes, int num_boxes,
                                        uint32_t salt, float texel, float step, float max_dist, const double* K,
                                        const double* R,
                                        const double* T, int width, int height, float* albedo, float* depth,
                                        float* normal, void* stream) {
  if (!hills || num_hills < 0 || num_hills > kMaxHills || (num_boxes > 0 && !boxes) || num_boxes < 0 || !K || !R ||
      !T || width <= 0 || height <= 0 || !albedo || !depth || !normal || !(texel > 0) || !(step > 0) ||
      !(max_dist > 0))
    return Fail(SMVS_EINVAL, "smvs_synth_render_aerial: bad arguments");
  SynthScene s;
  memset(&s, 0, sizeof(s));
  s.num_hills = num_hills;
  float hmin = 0.f, hmax = 0.f;
  for (int i = 0; i < num_hills; ++i) {
    for (int k = 0; k < 4; ++k) s.hills[i][k] = hills[4 * i + k];
    if (hills[4 * i + 2] > 0) hmax += hills[4 * i + 2]; else hmin += hills[4 * i + 2];
  }
  // Grid of 16 m cells over the boxes' extent.
  float bx0 = 0.f, by0 = 0.f, bx1 = 1.f, by1 = 1.f;
  for (int b = 0; b < num_boxes; ++b) {
    const float* B = boxes + 5 * b;
    if (b == 0 || B[0] < bx0) bx0 = B[0];
    if (b == 0 || B[1] < by0) by0 = B[1];
    if (b == 0 || B[2] > bx1) bx1 = B[2];
    if (b == 0 || B[3] > by1) by1 = B[3];
    hmax = std::max(hmax, B[4]);
  }
  s.z_lo = hmin - 0.5f;
  s.z_hi = hmax + 0.5f;
  s.cell = 16.f;
  s.grid_x0 = bx0;
  s.grid_y0 = by0;
  s.grid_nx = std::max(1, (int)std::ceil((bx1 - bx0) / s.cell));
  s.grid_ny = std::max(1, (int)std::ceil((by1 - by0) / s.cell));
  std::vector<std::vector<int>> cells((size_t)s.grid_nx * s.grid_ny);
  for (int b = 0; b < num_boxes; ++b) {
    const float* B = boxes + 5 * b;
    const int cx0 = std::max(0, (int)std::floor((B[0] - bx0) / s.cell));
    const int cy0 = std::max(0, (int)std::floor((B[1] - by0) / s.cell));
    const int cx1 = std::min(s.grid_nx - 1, (int)std::floor((B[2] - bx0) / s.cell));
    const int cy1 = std::min(s.grid_ny - 1, (int)std::floor((B[3] - by0) / s.cell));
    for (int cy = cy0; cy <= cy1; ++cy)
      for (int cx = cx0; cx <= cx1; ++cx) cells[(size_t)cy * s.grid_nx + cx].push_back(b);
  }
  std::vector<int> start(cells.size() + 1, 0), list;
  for (size_t c = 0; c < cells.size(); ++c) {
    start[c + 1] = start[c] + (int)cells[c].size();
    list.insert(list.end(), cells[c].begin(), cells[c].end());
  }
  if (list.empty()) list.push_back(0);
  std::vector<float> bx(boxes ? boxes : nullptr, boxes ? boxes + 5 * (size_t)num_boxes : nullptr);
  if (bx.empty()) bx.assign(5, 0.f);
  int* d_start = nullptr;
  int* d_list = nullptr;
  float* d_boxes = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMalloc(&d_start, start.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_list, list.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_boxes, bx.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(d_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_boxes, bx.data(), bx.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    s.cell_start = d_start;
    s.cell_boxes = d_list;
    s.boxes = d_boxes;
    s.salt = salt;
    SynthCamera cam;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        cam.R[3 * i + j] = (float)R[3 * i + j];
        cam.Rt[3 * i + j] = (float)R[3 * j + i];
      }
    for (int i = 0; i < 3; ++i)  // C = -R^T T (double)
      cam.C[i] = (float)(-(R[i] * T[0] + R[3 + i] * T[1] + R[6 + i] * T[2]));
    cam.iK[0] = (float)(1.0 / K[0]);
    cam.iK[1] = (float)(-K[2] / K[0]);
    cam.iK[2] = (float)(1.0 / K[4]);
    cam.iK[3] = (float)(-K[5] / K[4]);
    cam.W = width;
    cam.H = height;
    dim3 blk(32, 8), grd((width + 31) / 32, (height + 7) / 8);
    RenderAerialKernel<<<grd, blk, 0, st>>>(s, cam, texel, step, max_dist, albedo, depth, normal);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  cudaFree(d_start);
  cudaFree(d_list);
  cudaFree(d_boxes);
  if (e != cudaSuccess) return Fail(SMVS_ECUDA, cudaGetErrorString(e));
  return SMVS_OK;
}
