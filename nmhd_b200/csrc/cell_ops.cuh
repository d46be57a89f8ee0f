// Per-cell operations of one RK stage, shared by the single-box kernels
// (cell_stage.cu) and the batched-ensemble kernels (batch.cu), so that a box
// advanced in a batch is bitwise the box advanced alone.
//
// Cells are visited by 32 x 4 x 2 CTAs (x fastest).  Every periodic neighbour
// address is the cell address plus one of nine offsets computed once per
// thread.  Arithmetic follows the reference operation by operation
// (mhd_math.cuh); including files are compiled with -fmad=false.
#pragma once
#include "mhd_math.cuh"
#include "step.cuh"

namespace nmhd {
namespace cell {

constexpr int BX = 32, BY = 4, BZ = 2, kThreads = BX * BY * BZ;

__device__ __forceinline__ int wrap_any(int v, int s) {
  while (v < 0) v += s;
  while (v >= s) v -= s;
  return v;
}

// Offset from coordinate c to the periodic c + d.
__device__ __forceinline__ int woff(int c, int d, int s) { return wrap_any(c + d, s) - c; }

struct Offsets {
  int xm2, xm1, xp1, ym2, ym1, yp1, zm2, zm1, zp1;
};

__device__ __forceinline__ Offsets offsets(const GridParams &g, int x, int y, int z) {
  const int sxy = g.sx * g.sy;
  Offsets f;
  f.xm2 = woff(x, -2, g.sx);
  f.xm1 = woff(x, -1, g.sx);
  f.xp1 = woff(x, 1, g.sx);
  f.ym2 = woff(y, -2, g.sy) * g.sx;
  f.ym1 = woff(y, -1, g.sy) * g.sx;
  f.yp1 = woff(y, 1, g.sy) * g.sx;
  f.zm2 = woff(z, -2, g.sz) * sxy;
  f.zm1 = woff(z, -1, g.sz) * sxy;
  f.zp1 = woff(z, 1, g.sz) * sxy;
  return f;
}

// x / d for a grid spacing d; with power-of-two spacings the product with the
// exact reciprocal is the same float.
template <bool kPow2>
__device__ __forceinline__ float divs(float x, float d, float inv) {
  return kPow2 ? x * inv : x / d;
}

// Time step of the current step: min(goal, CFL), clamped to the goal
// (src/library/mhd_solver.inlrb:870-901).
__device__ __forceinline__ float step_dt(const StepCtl *c, bool *last) {
  if (c->dt_seq) {
    if (last) *last = false;
    return c->dt_seq[c->generation - c->dt_seq_base];
  }
  const float cmin = __uint_as_float(c->cfl_cur);
  float dt = fminf(c->goal, cmin);
  const double next_time = c->time + (double)dt;
  const bool l = next_time > (double)c->goal;
  if (l) dt = (float)((double)c->goal - c->time);
  if (last) *last = l;
  return dt;
}

// Loads of face_flux's inputs: read-only global memory (the stage input in
// HBM) or a plain load (a shared-memory copy of it).
struct GlobalLd {
  __device__ static __forceinline__ float ld(const float *p) { return __ldg(p); }
};
struct SharedLd {
  __device__ static __forceinline__ float ld(const float *p) { return *p; }
};

// Flux through the lower face of cell o along runtime axis `ax` (one HLLD
// instance serves all three axes).  The inputs are read at w + f*NW + o + d
// (field f, stencil offset d): m2, m1, p1 are the offsets of the stencil
// cells -2, -1, +1 along ax; t1, t2 the +1 offsets along the transverse axes
// ax+1 and ax+2 (mod 3).  The 7 results go to flux + (7*ax + k)*N + oo:
// mass, momentum x/y/z (absolute components), energy, F(B_t1), F(B_t2)
// (calc_flux_kernel<EX>, src/library/mhd_solver.inlrb:562-636).
template <class L = GlobalLd, class S = size_t>
__device__ __forceinline__ void face_flux(const GridParams &g, const float *__restrict__ w, S NW, int o, int ax,
                                          int m2, int m1, int p1, int t1, int t2, int yidx, float dt,
                                          float *__restrict__ flux, size_t N, int oo) {
  const int e1 = ax == 2 ? 0 : ax + 1, e2 = ax == 0 ? 2 : ax - 1;
  const float *rho = w, *p = w + 4 * NW;
  const float *vn = w + (1 + ax) * NW, *v1 = w + (1 + e1) * NW, *v2 = w + (1 + e2) * NW;
  const float *bn = w + (5 + ax) * NW, *b1 = w + (5 + e1) * NW, *b2 = w + (5 + e2) * NW;
  const int s[4] = {m2, m1, 0, p1};
  float bc1[4], bc2[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int c = o + s[t];
    bc1[t] = 0.5f * (L::ld(b1 + c) + L::ld(b1 + c + t1));
    bc2[t] = 0.5f * (L::ld(b2 + c) + L::ld(b2 + c + t2));
  }
  HlldIn in;
  if (g.order2) {
    reconstruct4(L::ld(rho + o + m2), L::ld(rho + o + m1), L::ld(rho + o), L::ld(rho + o + p1), in.dl, in.dr);
    reconstruct4(L::ld(vn + o + m2), L::ld(vn + o + m1), L::ld(vn + o), L::ld(vn + o + p1), in.ul, in.ur);
    reconstruct4(L::ld(v1 + o + m2), L::ld(v1 + o + m1), L::ld(v1 + o), L::ld(v1 + o + p1), in.vl, in.vr);
    reconstruct4(L::ld(v2 + o + m2), L::ld(v2 + o + m1), L::ld(v2 + o), L::ld(v2 + o + p1), in.wl, in.wr);
    reconstruct4(L::ld(p + o + m2), L::ld(p + o + m1), L::ld(p + o), L::ld(p + o + p1), in.pl, in.pr);
    reconstruct4(bc1[0], bc1[1], bc1[2], bc1[3], in.byl, in.byr);
    reconstruct4(bc2[0], bc2[1], bc2[2], bc2[3], in.bzl, in.bzr);
  } else {
    in.dl = L::ld(rho + o + m1); in.dr = L::ld(rho + o);
    in.ul = L::ld(vn + o + m1); in.ur = L::ld(vn + o);
    in.vl = L::ld(v1 + o + m1); in.vr = L::ld(v1 + o);
    in.wl = L::ld(v2 + o + m1); in.wr = L::ld(v2 + o);
    in.pl = L::ld(p + o + m1); in.pr = L::ld(p + o);
    in.byl = bc1[1]; in.byr = bc1[2];
    in.bzl = bc2[1]; in.bzr = bc2[2];
  }
  if (g.shear) {
    // face-centred Kepler acceleration, half a stage kick on the normal velocity
    float acc;
    if (ax == 0) {
      const float vY = 0.5f * (L::ld(w + 2 * NW + o + m1) + L::ld(w + 2 * NW + o));
      acc = -2.0f * g.omega * vY;
    } else if (ax == 1) {
      const float vX = 0.5f * (L::ld(w + NW + o + m1) + L::ld(w + NW + o));
      acc = 2.0f * g.omega * vX + 2.0f * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((float)yidx + 0.5f));
    } else {
      acc = 0.0f;
    }
    const float mbv = 0.5f * dt * acc;
    in.ul += mbv;
    in.ur += mbv;
  }
  float f[7];
  hlld_flux(g.gamma, L::ld(bn + o), in, f);
  float *out = flux + (size_t)(7 * ax) * N + oo;
  out[0] = f[0];
  out[(1 + ax) * N] = f[1];
  out[(1 + e1) * N] = f[2];
  out[(1 + e2) * N] = f[3];
  out[4 * N] = f[4];
  out[5 * N] = f[5];
  out[6 * N] = f[6];
}

// The three lower-face fluxes of cell (x, y, z) (inside the box).
__device__ __forceinline__ void flux_cell(const GridParams &g, const float *__restrict__ w,
                                          float *__restrict__ flux, int x, int y, int z, float dt) {
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const Offsets f = offsets(g, x, y, z);
#pragma unroll 1
  for (int ax = 0; ax < 3; ++ax) {
    const int m2 = ax == 0 ? f.xm2 : ax == 1 ? f.ym2 : f.zm2;
    const int m1 = ax == 0 ? f.xm1 : ax == 1 ? f.ym1 : f.zm1;
    const int p1 = ax == 0 ? f.xp1 : ax == 1 ? f.yp1 : f.zp1;
    const int t1 = ax == 0 ? f.yp1 : ax == 1 ? f.zp1 : f.xp1;
    const int t2 = ax == 0 ? f.zp1 : ax == 1 ? f.xp1 : f.yp1;
    face_flux(g, w, N, o, ax, m2, m1, p1, t1, t2, y, dt, flux, N, o);
  }
}

// Upwind choice of corner_magnet_flux (src/library/mhd_solver.inlrb:641-653)
// for the wind sum w of the four cell velocities around an edge: f0 (the flux
// one step down the wind axis) for w > 0, f1 for w < 0, their mean at a tie.
__device__ __forceinline__ float upwind(float w, float f0, float f1) {
  return w > 0.0f ? f0 : (w < 0.0f ? f1 : 0.5f * (f0 + f1));
}

// Sources of the constrained-transport inputs around one cell: velocity
// component c (0..2) and B flux k (0..5: F_x(B_y), F_x(B_z), F_y(B_z),
// F_y(B_x), F_z(B_x), F_z(B_y)) of the neighbour (dx, dy, dz), each in -1..1.
// CtGlobal and CtGlobalLean read HBM through the periodic neighbour offsets
// of the cell.
struct CtGlobal {
  const float *v[3];
  const float *f[6];
  int xm, xp, ym, yp, zm, zp;
  __device__ __forceinline__ int off(int dx, int dy, int dz) const {
    return (dx < 0 ? xm : dx > 0 ? xp : 0) + (dy < 0 ? ym : dy > 0 ? yp : 0) + (dz < 0 ? zm : dz > 0 ? zp : 0);
  }
  __device__ __forceinline__ float vel(int c, int dx, int dy, int dz) const { return __ldg(v[c] + off(dx, dy, dz)); }
  __device__ __forceinline__ float flx(int k, int dx, int dy, int dz) const { return __ldg(f[k] + off(dx, dy, dz)); }
};

__device__ __forceinline__ CtGlobal ct_global(const GridParams &g, const float *win, const float *flux, int x,
                                              int y, int z) {
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const Offsets f = offsets(g, x, y, z);
  CtGlobal s;
  s.v[0] = win + N + o;
  s.v[1] = win + 2 * N + o;
  s.v[2] = win + 3 * N + o;
  s.f[0] = flux + 5 * N + o;
  s.f[1] = flux + 6 * N + o;
  s.f[2] = flux + 12 * N + o;
  s.f[3] = flux + 13 * N + o;
  s.f[4] = flux + 19 * N + o;
  s.f[5] = flux + 20 * N + o;
  s.xm = f.xm1;
  s.xp = f.xp1;
  s.ym = f.ym1;
  s.yp = f.yp1;
  s.zm = f.zm1;
  s.zp = f.zp1;
  return s;
}

// The same inputs for a cell whose neighbours need no periodic wrap: x
// neighbours at constant offsets, y and z ones at +-Sx and +-Sx*Sy.
struct CtInterior {
  const float *v[3];
  const float *f[6];
  int sx, sxy;
  __device__ __forceinline__ int off(int dx, int dy, int dz) const { return dx + dy * sx + dz * sxy; }
  __device__ __forceinline__ float vel(int c, int dx, int dy, int dz) const { return __ldg(v[c] + off(dx, dy, dz)); }
  __device__ __forceinline__ float flx(int k, int dx, int dy, int dz) const { return __ldg(f[k] + off(dx, dy, dz)); }
};

__device__ __forceinline__ CtInterior ct_interior(const GridParams &g, const float *win, const float *flux, int o) {
  const size_t N = (size_t)g.n;
  CtInterior s;
  s.v[0] = win + N + o;
  s.v[1] = win + 2 * N + o;
  s.v[2] = win + 3 * N + o;
  s.f[0] = flux + 5 * N + o;
  s.f[1] = flux + 6 * N + o;
  s.f[2] = flux + 12 * N + o;
  s.f[3] = flux + 13 * N + o;
  s.f[4] = flux + 19 * N + o;
  s.f[5] = flux + 20 * N + o;
  s.sx = g.sx;
  s.sxy = g.sx * g.sy;
  return s;
}

// The same inputs through two base pointers (fewer live registers: the
// batched kernels, which inline both spacing variants, spill less with it).
struct CtGlobalLean {
  const float *win, *flux;  // the stage input and the flux scratch, at cell o
  size_t N;
  int xm, xp, ym, yp, zm, zp;
  __device__ __forceinline__ int off(int dx, int dy, int dz) const {
    return (dx < 0 ? xm : dx > 0 ? xp : 0) + (dy < 0 ? ym : dy > 0 ? yp : 0) + (dz < 0 ? zm : dz > 0 ? zp : 0);
  }
  __device__ __forceinline__ float vel(int c, int dx, int dy, int dz) const {
    return __ldg(win + (1 + c) * N + off(dx, dy, dz));
  }
  __device__ __forceinline__ float flx(int k, int dx, int dy, int dz) const {
    // F_x(B_y), F_x(B_z), F_y(B_z), F_y(B_x), F_z(B_x), F_z(B_y): fields 5, 6, 12, 13, 19, 20
    return __ldg(flux + (5 + (k >> 1) * 7 + (k & 1)) * N + off(dx, dy, dz));
  }
};

__device__ __forceinline__ CtGlobalLean ct_global_lean(const GridParams &g, const float *win, const float *flux, int x,
                                              int y, int z) {
  const int o = (z * g.sy + y) * g.sx + x;
  const Offsets f = offsets(g, x, y, z);
  CtGlobalLean s;
  s.win = win + o;
  s.flux = flux + o;
  s.N = (size_t)g.n;
  s.xm = f.xm1;
  s.xp = f.xp1;
  s.ym = f.ym1;
  s.yp = f.yp1;
  s.zm = f.zm1;
  s.zp = f.zp1;
  return s;
}

// Constrained transport of one stage (add_flux_kernel's B part,
// mhd_solver.inlrb:695-712, summed over the x, y, z sweeps in that order):
// new face B on the lower x-, y- and z-face of cell o, written into wo.  The
// 18 corner fluxes (corner(), at the cell's edges and one step up each
// in-plane axis) read 39 distinct velocities and 30 distinct fluxes; each is
// read once and every wind sum keeps corner()'s order.
template <bool kPow2, class Src>
__device__ __forceinline__ void ct_core(const GridParams &g, const Src &S, const float *__restrict__ wb,
                                        float *__restrict__ wo, int o, float dt) {
  const size_t N = (size_t)g.n;
  // velocities around the cell
  const float x_0 = S.vel(0, 0, 0, 0), x_xm = S.vel(0, -1, 0, 0), x_ym = S.vel(0, 0, -1, 0);
  const float x_ymxm = S.vel(0, -1, -1, 0), x_yp = S.vel(0, 0, 1, 0), x_ypxm = S.vel(0, -1, 1, 0);
  const float x_xp = S.vel(0, 1, 0, 0), x_xpym = S.vel(0, 1, -1, 0), x_zm = S.vel(0, 0, 0, -1);
  const float x_zmxm = S.vel(0, -1, 0, -1), x_zp = S.vel(0, 0, 0, 1), x_zpxm = S.vel(0, -1, 0, 1);
  const float x_xpzm = S.vel(0, 1, 0, -1);
  const float y_0 = S.vel(1, 0, 0, 0), y_ym = S.vel(1, 0, -1, 0), y_xm = S.vel(1, -1, 0, 0);
  const float y_xmym = S.vel(1, -1, -1, 0), y_yp = S.vel(1, 0, 1, 0), y_ypxm = S.vel(1, -1, 1, 0);
  const float y_xp = S.vel(1, 1, 0, 0), y_xpym = S.vel(1, 1, -1, 0), y_zm = S.vel(1, 0, 0, -1);
  const float y_zmym = S.vel(1, 0, -1, -1), y_zp = S.vel(1, 0, 0, 1), y_zpym = S.vel(1, 0, -1, 1);
  const float y_ypzm = S.vel(1, 0, 1, -1);
  const float z_0 = S.vel(2, 0, 0, 0), z_zm = S.vel(2, 0, 0, -1), z_xm = S.vel(2, -1, 0, 0);
  const float z_xmzm = S.vel(2, -1, 0, -1), z_zp = S.vel(2, 0, 0, 1), z_zpxm = S.vel(2, -1, 0, 1);
  const float z_xp = S.vel(2, 1, 0, 0), z_xpzm = S.vel(2, 1, 0, -1), z_ym = S.vel(2, 0, -1, 0);
  const float z_ymzm = S.vel(2, 0, -1, -1), z_zpym = S.vel(2, 0, -1, 1), z_yp = S.vel(2, 0, 1, 0);
  const float z_ypzm = S.vel(2, 0, 1, -1);
  // B fluxes
  const float xy_0 = S.flx(0, 0, 0, 0), xy_ym = S.flx(0, 0, -1, 0), xy_yp = S.flx(0, 0, 1, 0);
  const float xy_xp = S.flx(0, 1, 0, 0), xy_xpym = S.flx(0, 1, -1, 0);
  const float xz_0 = S.flx(1, 0, 0, 0), xz_zm = S.flx(1, 0, 0, -1), xz_zp = S.flx(1, 0, 0, 1);
  const float xz_xp = S.flx(1, 1, 0, 0), xz_xpzm = S.flx(1, 1, 0, -1);
  const float yz_0 = S.flx(2, 0, 0, 0), yz_zm = S.flx(2, 0, 0, -1), yz_zp = S.flx(2, 0, 0, 1);
  const float yz_yp = S.flx(2, 0, 1, 0), yz_ypzm = S.flx(2, 0, 1, -1);
  const float yx_0 = S.flx(3, 0, 0, 0), yx_xm = S.flx(3, -1, 0, 0), yx_yp = S.flx(3, 0, 1, 0);
  const float yx_ypxm = S.flx(3, -1, 1, 0), yx_xp = S.flx(3, 1, 0, 0);
  const float zx_0 = S.flx(4, 0, 0, 0), zx_xm = S.flx(4, -1, 0, 0), zx_zp = S.flx(4, 0, 0, 1);
  const float zx_zpxm = S.flx(4, -1, 0, 1), zx_xp = S.flx(4, 1, 0, 0);
  const float zy_0 = S.flx(5, 0, 0, 0), zy_ym = S.flx(5, 0, -1, 0), zy_zp = S.flx(5, 0, 0, 1);
  const float zy_zpym = S.flx(5, 0, -1, 1), zy_yp = S.flx(5, 0, 1, 0);
  // corner(vb, fb, e, mb, ma): wind vb[e] + vb[e+mb] + vb[e+ma] + vb[e+ma+mb],
  // f0 = fb[e+mb], f1 = fb[e]
  const float XY00 = upwind(y_0 + y_ym + y_xm + y_xmym, xy_ym, xy_0);            // F_x(B_y), wind v_y
  const float XY01 = upwind(y_yp + y_0 + y_ypxm + y_xm, xy_0, xy_yp);
  const float XY10 = upwind(y_xp + y_xpym + y_0 + y_ym, xy_xpym, xy_xp);
  const float YX00 = upwind(x_0 + x_xm + x_ym + x_ymxm, yx_xm, yx_0);            // F_y(B_x), wind v_x
  const float YX01 = upwind(x_yp + x_ypxm + x_0 + x_xm, yx_ypxm, yx_yp);
  const float YX10 = upwind(x_xp + x_0 + x_xpym + x_ym, yx_0, yx_xp);
  const float XZ00 = upwind(z_0 + z_zm + z_xm + z_xmzm, xz_zm, xz_0);            // F_x(B_z), wind v_z
  const float XZ01 = upwind(z_zp + z_0 + z_zpxm + z_xm, xz_0, xz_zp);
  const float XZ10 = upwind(z_xp + z_xpzm + z_0 + z_zm, xz_xpzm, xz_xp);
  const float ZX00 = upwind(x_0 + x_xm + x_zm + x_zmxm, zx_xm, zx_0);            // F_z(B_x), wind v_x
  const float ZX01 = upwind(x_zp + x_zpxm + x_0 + x_xm, zx_zpxm, zx_zp);
  const float ZX10 = upwind(x_xp + x_0 + x_xpzm + x_zm, zx_0, zx_xp);
  const float YZ00 = upwind(z_0 + z_zm + z_ym + z_ymzm, yz_zm, yz_0);            // F_y(B_z), wind v_z
  const float YZ01 = upwind(z_zp + z_0 + z_zpym + z_ym, yz_0, yz_zp);
  const float YZ10 = upwind(z_yp + z_ypzm + z_0 + z_zm, yz_ypzm, yz_yp);
  const float ZY00 = upwind(y_0 + y_ym + y_zm + y_zmym, zy_ym, zy_0);            // F_z(B_y), wind v_y
  const float ZY01 = upwind(y_zp + y_zpym + y_0 + y_ym, zy_zpym, zy_zp);
  const float ZY10 = upwind(y_yp + y_0 + y_ypzm + y_zm, zy_0, zy_yp);
  const float dx = g.dx, dy = g.dy, dz = g.dz, ix = g.inv_dx, iy = g.inv_dy, iz = g.inv_dz;
  float pb = 0.0f;
  pb = pb + 0.5f * (divs<kPow2>(XY01 - XY00, dy, iy) + divs<kPow2>(XZ01 - XZ00, dz, iz));
  pb = pb - divs<kPow2>(0.5f * (YX01 - YX00), dy, iy);
  pb = pb - divs<kPow2>(0.5f * (ZX01 - ZX00), dz, iz);
  wo[5 * N + o] = wb[5 * N + o] + dt * pb;
  pb = 0.0f;
  pb = pb - divs<kPow2>(0.5f * (XY10 - XY00), dx, ix);
  pb = pb + 0.5f * (divs<kPow2>(YZ01 - YZ00, dz, iz) + divs<kPow2>(YX10 - YX00, dx, ix));
  pb = pb - divs<kPow2>(0.5f * (ZY01 - ZY00), dz, iz);
  wo[6 * N + o] = wb[6 * N + o] + dt * pb;
  pb = 0.0f;
  pb = pb - divs<kPow2>(0.5f * (XZ10 - XZ00), dx, ix);
  pb = pb - divs<kPow2>(0.5f * (YZ10 - YZ00), dy, iy);
  pb = pb + 0.5f * (divs<kPow2>(ZX10 - ZX00, dx, ix) + divs<kPow2>(ZY10 - ZY00, dy, iy));
  wo[7 * N + o] = wb[7 * N + o] + dt * pb;
}

// Rest of the stage for cell (x, y, z): flux divergence of rho, m, E
// (mhd_solver.inlrb:689-693), conserved state before the stage (to_conserved
// :762-777), update (add_pace/update :797-835), primitive recovery with the new
// face B (:779-795) and the Kepler kick (:837-848).  In the final stage returns
// the cell's CFL time (inf for margin cells, which the margin kernel covers)
// and sets *bad for a non-physical result.
template <bool kPow2>
__device__ __forceinline__ float prim_cell(const GridParams &g, const float *__restrict__ wb,
                                           float *__restrict__ wo, const float *__restrict__ flux, int x,
                                           int y, int z, float dt, bool final_stage, int *bad) {
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const int xp = x + 1 < g.sx ? 1 : 1 - g.sx;
  const int yp = (y + 1 < g.sy ? 1 : 1 - g.sy) * g.sx;
  const int zp = (z + 1 < g.sz ? 1 : 1 - g.sz) * g.sx * g.sy;
  const float *Fx = flux, *Fy = flux + 7 * N, *Fz = flux + 14 * N;
  // all loads first: 30 face fluxes
  float fl[5][6];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    fl[v][0] = __ldg(Fx + v * N + o);
    fl[v][1] = __ldg(Fx + v * N + o + xp);
    fl[v][2] = __ldg(Fy + v * N + o);
    fl[v][3] = __ldg(Fy + v * N + o + yp);
    fl[v][4] = __ldg(Fz + v * N + o);
    fl[v][5] = __ldg(Fz + v * N + o + zp);
  }
  float pace[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    float pc = 0.0f;
    pc = pc + divs<kPow2>(fl[v][0] - fl[v][1], g.dx, g.inv_dx);
    pc = pc + divs<kPow2>(fl[v][2] - fl[v][3], g.dy, g.inv_dy);
    pc = pc + divs<kPow2>(fl[v][4] - fl[v][5], g.dz, g.inv_dz);
    pace[v] = pc;
  }
  const float gm1 = g.gamma - 1.0f;
  const float rho0 = wb[o];
  const float vx0 = wb[N + o], vy0 = wb[2 * N + o], vz0 = wb[3 * N + o], p0 = wb[4 * N + o];
  const float bxl = wb[5 * N + o], bxh = wb[5 * N + o + xp];
  const float byl = wb[6 * N + o], byh = wb[6 * N + o + yp];
  const float bzl = wb[7 * N + o], bzh = wb[7 * N + o + zp];
  const float mx0 = rho0 * vx0, my0 = rho0 * vy0, mz0 = rho0 * vz0;
  const float e0 = p0 / gm1 + 0.5f * rho0 * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0) +
                   0.25f * (bxl * bxl + bxh * bxh + byl * byl + byh * byh + bzl * bzl + bzh * bzh);
  const float rho = rho0 + dt * pace[0];
  const float mx = mx0 + dt * pace[1];
  const float my = my0 + dt * pace[2];
  const float mz = mz0 + dt * pace[3];
  const float ene = e0 + dt * pace[4];
  // new face B from the CT pass (this cell's lower faces and its neighbours')
  const float bx0 = wo[5 * N + o], bx1 = wo[5 * N + o + xp];
  const float by0 = wo[6 * N + o], by1 = wo[6 * N + o + yp];
  const float bz0 = wo[7 * N + o], bz1 = wo[7 * N + o + zp];
  float vxo = mx / rho, vyo = my / rho, vzo = mz / rho;
  const float eint = ene - 0.5f * (mx * mx + my * my + mz * mz) / rho -
                     0.25f * (bx0 * bx0 + bx1 * bx1 + by0 * by0 + by1 * by1 + bz0 * bz0 + bz1 * bz1);
  const float po = eint * gm1;
  if (g.shear) {
    const float ax = -2.0f * g.omega * vyo;
    const float ay = 2.0f * g.omega * vxo + 2.0f * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((float)y + 0.5f));
    vxo = vxo + dt * ax;
    vyo = vyo + dt * ay;
    vzo = vzo + dt * 0.0f;
  }
  wo[o] = rho;
  wo[N + o] = vxo;
  wo[2 * N + o] = vyo;
  wo[3 * N + o] = vzo;
  wo[4 * N + o] = po;
  float tcfl = __uint_as_float(0x7f800000u);
  if (final_stage) {
    *bad = !(rho > 0.0f) || !(po > 0.0f) || !isfinite(vxo) || !isfinite(vyo) || !isfinite(vzo) ||
           !isfinite(bx0) || !isfinite(by0) || !isfinite(bz0);
    const bool margin_cell = (y < g.my) || (y >= g.sy - g.my) || (g.mz > 0 && (z < g.mz || z >= g.sz - g.mz - 1));
    if (!margin_cell) {
      // cfl_condition_inner/kernel (mhd_solver.inlrb:496-521)
      const float b2 = fmaxf(bx0 * bx0, bx1 * bx1) + fmaxf(by0 * by0, by1 * by1) + fmaxf(bz0 * bz0, bz1 * bz1);
      const float cs = sqrtf((g.gamma * po + b2) / rho);
      tcfl = fminf(fminf(g.cfl * g.dx / fabsf(vxo + cs), g.cfl * g.dy / fabsf(vyo + cs)),
                   g.cfl * g.dz / fabsf(vzo + cs));
    }
  }
  return tcfl;
}

__device__ __forceinline__ float block_min(float v, float *red) {
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tid = (threadIdx.z * BY + threadIdx.y) * BX + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < kThreads / 32 ? red[lane] : __uint_as_float(0x7f800000u);
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  __syncthreads();
  return v;
}

// End of one tile of a final stage (called by every thread of the CTA): fold
// the tile's CFL minimum and status into the box's control block; the last
// of the box's `ntiles` tiles advances the box's clock (GlobalSetup::proceed,
// mhd_solver.inlrb:981), rotates the state buffers and the CFL accumulators.
__device__ __forceinline__ void finish_tile(StepCtl *ctl, unsigned ntiles, float tcfl, int bad, float *dt_hist,
                                            float *red) {
  tcfl = block_min(tcfl, red);
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    atomicMin(&ctl->cfl_next, __float_as_uint(tcfl));
    if (bad) atomicOr(&ctl->status, kStatusNumerical);
    __threadfence();
    const unsigned prev = atomicAdd(&ctl->blocks_done, 1u);
    if (prev == ntiles - 1) {
      __threadfence();
      bool last;
      const float dts = step_dt(ctl, &last);
      volatile StepCtl *vc = ctl;
      const long long gen = vc->generation;
      dt_hist[gen % kDtHistCap] = dts;
      vc->time = vc->time + (double)dts;
      vc->generation = gen + 1;
      vc->parity = vc->parity ^ 1;
      vc->cfl_cur = atomicAdd(&ctl->cfl_next, 0u);
      vc->cfl_next = 0x7f800000u;
      if (!(dts >= 0.0f)) atomicOr(&ctl->status, kStatusBadDt);
      if (last || vc->status) vc->done = 1;
      vc->blocks_done = 0;
    }
  }
}

__device__ __forceinline__ const float *pick(const StepCtl *c, int sel, const float *w0, const float *w1,
                                             const float *wp) {
  if (sel == 2) return wp;
  return (sel == 0) == (c->parity == 0) ? w0 : w1;
}

// Buffer index (0 w0, 1 w1, 2 predictor) that pick() selects.
__device__ __forceinline__ int pick_index(const StepCtl *c, int sel) {
  if (sel == 2) return 2;
  return (sel == 0) == (c->parity == 0) ? 0 : 1;
}

}  // namespace cell
}  // namespace nmhd
