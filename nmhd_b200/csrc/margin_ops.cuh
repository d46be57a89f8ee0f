// Margin fill and CFL-time operations shared by the single-box kernels
// (step.cu) and the batched-ensemble kernels (batch.cu).
#pragma once
#include <cuda_runtime.h>

#include "step.cuh"

namespace nmhd {
namespace margin {

__device__ __forceinline__ int wrap(int v, int s) {
  while (v < 0) v += s;
  while (v >= s) v -= s;
  return v;
}

// CFL time of cell (x, y, z) (cfl_condition_inner/kernel,
// src/library/mhd_solver.inlrb:496-521): min over axes of
// cfl*d / |v_d + sqrt((gamma p + b2)/rho)|, b2 = sum of max(B_lo^2, B_hi^2).
__device__ __forceinline__ float cfl_of_cell(const GridParams &g, const float *w, int x, int y, int z) {
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const int oxp = (z * g.sy + y) * g.sx + wrap(x + 1, g.sx);
  const int oyp = (z * g.sy + wrap(y + 1, g.sy)) * g.sx + x;
  const int ozp = (wrap(z + 1, g.sz) * g.sy + y) * g.sx + x;
  const float bxl = w[5 * N + o], bxh = w[5 * N + oxp];
  const float byl = w[6 * N + o], byh = w[6 * N + oyp];
  const float bzl = w[7 * N + o], bzh = w[7 * N + ozp];
  const float b2 = fmaxf(bxl * bxl, bxh * bxh) + fmaxf(byl * byl, byh * byh) + fmaxf(bzl * bzl, bzh * bzh);
  const float c = sqrtf((g.gamma * w[4 * N + o] + b2) / w[o]);
  const float tx = g.cfl * g.dx / fabsf(w[N + o] + c);
  const float ty = g.cfl * g.dy / fabsf(w[2 * N + o] + c);
  const float tz = g.cfl * g.dz / fabsf(w[3 * N + o] + c);
  return fminf(fminf(tx, ty), tz);
}

// Number of cells whose CFL time the margin pass covers: the Y-margin rows, and
// with Z margins the Z-margin planes plus the last interior plane (its upper
// z-face is rewritten by the Z copy).  The final stage covers all other cells.
__device__ __host__ __forceinline__ long long margin_cfl_cells(const GridParams &g) {
  return 2LL * g.my * g.sx * g.sz + (g.mz > 0 ? (2LL * g.mz + 1) * g.sx * g.sy : 0);
}

__device__ __forceinline__ void margin_cfl_cell(const GridParams &g, int idx, int *x, int *y, int *z) {
  const int part_a = 2 * g.my * g.sx * g.sz;
  if (idx < part_a) {
    *x = idx % g.sx;
    const int r = (idx / g.sx) % (2 * g.my);
    *z = idx / (g.sx * 2 * g.my);
    *y = r < g.my ? r : g.sy - 2 * g.my + r;
  } else {
    const int j = idx - part_a;
    *x = j % g.sx;
    *y = (j / g.sx) % g.sy;
    const int p = j / (g.sx * g.sy);
    *z = p < g.mz ? p : g.sz - g.mz - 1 + (p - g.mz);
  }
}

// Integer and fractional shear displacement of the Y-margin exchange at time t
// (relative_displacement, src/library/mhd_solver.inlrb:244-259): all double
// except the float product fold * kExtentX.
struct ShearShift {
  int dint;
  float f;
};
__device__ __forceinline__ ShearShift shear_shift(const GridParams &g, double time) {
  const double d0 = 0.0 + time * g.rel_vel;
  const int fold = (int)floor(d0 / (double)g.extent_x);
  const double d1 = d0 - (double)((float)fold * g.extent_x);
  ShearShift s;
  s.dint = (int)floor(d1 / (double)g.dx);
  s.f = (float)(d1 / (double)g.dx - s.dint);
  return s;
}

// Gather half of the Y-margin exchange for item idx = (sz*M + sy)*Sx + sx,
// sy < M (communicate_gather_kernel_y, mhd_solver.inlrb:184-222): field v of
// the top interior row Sy-2M+sy shifted by +d_int in x with vx -
// relative_velocity (`inc`, sent to the rank above) and of the bottom interior
// row M+sy shifted by -d_int-1 with vx + relative_velocity (`dec`, sent to the
// rank below).  The reference's two-point interpolation weights both multiply
// the same sample; that arithmetic is kept.
__device__ __forceinline__ void gather_y_item(const GridParams &g, const ShearShift &sh, const float *w,
                                              int idx, float inc[8], float dec[8]) {
  const int M = g.my;
  const int sx = idx % g.sx;
  const int sy = (idx / g.sx) % M;
  const int sz = idx / (g.sx * M);
  const float rv = (float)g.rel_vel;
  const int inc_x = wrap((sx + sh.dint) % g.sx, g.sx);
  const int dec_x = wrap((sx - sh.dint - 1) % g.sx, g.sx);
  const size_t N = (size_t)g.n;
  const int src_inc = (sz * g.sy + (g.sy - 2 * M + sy)) * g.sx + inc_x;
  const int src_dec = (sz * g.sy + (M + sy)) * g.sx + dec_x;
  const float omf = 1.0f - sh.f;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const float vi = w[v * N + src_inc];
    const float vd = w[v * N + src_dec];
    float bi = omf * vi + sh.f * vi;
    float bd = sh.f * vd + omf * vd;
    if (v == 1) {
      bi = bi - rv;
      bd = bd + rv;
    }
    inc[v] = bi;
    dec[v] = bd;
  }
}

// Scatter half (communicate_scatter_kernel_y, mhd_solver.inlrb:224-242): the
// bottom margin row sy takes `inc` (from the rank below), the top margin row
// Sy-M+sy takes `dec` (from the rank above); By of row Sy-M (the interior's
// upper face) is kept.
__device__ __forceinline__ void scatter_y_item(const GridParams &g, float *w, int idx, const float inc[8],
                                               const float dec[8]) {
  const int M = g.my;
  const int sx = idx % g.sx;
  const int sy = (idx / g.sx) % M;
  const int sz = idx / (g.sx * M);
  const size_t N = (size_t)g.n;
  const int dst_lo = (sz * g.sy + sy) * g.sx + sx;
  const int dst_hi = (sz * g.sy + (g.sy - M + sy)) * g.sx + sx;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    w[v * N + dst_lo] = inc[v];
    if (!(v == 6 && sy == 0)) w[v * N + dst_hi] = dec[v];
  }
}

// One item of the shearing-periodic Y-margin fill of a single box (one rank:
// every message of the exchange goes to itself).  Reads only interior rows and
// writes only margin rows, so it runs in place.
__device__ __forceinline__ void fill_y_item(const GridParams &g, double time, float *w, int idx) {
  float inc[8], dec[8];
  gather_y_item(g, shear_shift(g, time), w, idx, inc, dec);
  scatter_y_item(g, w, idx, inc, dec);
}

}  // namespace margin
}  // namespace nmhd
