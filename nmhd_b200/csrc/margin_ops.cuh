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

// One item (sx, sy, sz), sy < M, of the shearing-periodic Y-margin fill
// (communicate_gather/scatter_kernel_y, mhd_solver.inlrb:184-242, with
// relative_displacement :244-259) for one rank: the bottom margin row sy takes
// the top interior row Sy-2M+sy shifted by +d_int in x with vx - rel_vel; the
// top margin row Sy-M+sy takes the bottom interior row M+sy shifted by
// -d_int-1 with vx + rel_vel; By of row Sy-M is kept.  The reference's
// two-point interpolation weights both multiply the same sample; that
// arithmetic is kept.
__device__ __forceinline__ void fill_y_item(const GridParams &g, double time, float *w, int idx) {
  const int M = g.my;
  const int sx = idx % g.sx;
  const int sy = (idx / g.sx) % M;
  const int sz = idx / (g.sx * M);
  // relative_displacement(t): all double except the float product fold*kExtentX
  const double d0 = 0.0 + time * g.rel_vel;
  const int fold = (int)floor(d0 / (double)g.extent_x);
  const double d1 = d0 - (double)((float)fold * g.extent_x);
  const int dint = (int)floor(d1 / (double)g.dx);
  const float f = (float)(d1 / (double)g.dx - dint);
  const float rv = (float)g.rel_vel;
  const int inc_x = wrap((sx + dint) % g.sx, g.sx);
  const int dec_x = wrap((sx - dint - 1) % g.sx, g.sx);
  const size_t N = (size_t)g.n;
  const int src_inc = (sz * g.sy + (g.sy - 2 * M + sy)) * g.sx + inc_x;
  const int src_dec = (sz * g.sy + (M + sy)) * g.sx + dec_x;
  const int dst_lo = (sz * g.sy + sy) * g.sx + sx;
  const int dst_hi = (sz * g.sy + (g.sy - M + sy)) * g.sx + sx;
  const float omf = 1.0f - f;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const float vi = w[v * N + src_inc];
    const float vd = w[v * N + src_dec];
    float bi = omf * vi + f * vi;
    float bd = f * vd + omf * vd;
    if (v == 1) {
      bi = bi - rv;
      bd = bd + rv;
    }
    w[v * N + dst_lo] = bi;
    if (!(v == 6 && sy == 0)) w[v * N + dst_hi] = bd;
  }
}

}  // namespace margin
}  // namespace nmhd
