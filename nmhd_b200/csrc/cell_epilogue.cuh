// Fused stage epilogue of the per-cell kernels: constrained transport and the
// conserved update of one RK stage in one pass over a 32 x 4 x 2-cell tile
// (add_flux_kernel's B part, src/library/mhd_solver.inlrb:641-714, then
// :689-693, 762-848 and, in the final stage, the CFL reduction :496-521).
//
// The tile stages the stage input's velocities and the six B-flux fields of
// the face-flux scratch, each with the halo the tile's edges need, in shared
// memory; computes every corner EMF of the tile's edges ONCE (the per-cell
// form recomputes each of them at up to four cells); from them the new face B
// of the tile's cells and of the upper halo faces (bx at x0+32, by at y0+4,
// bz at z0+2); then each thread finishes its cell from shared memory: flux
// divergence, conserved update, primitive recovery with the new B, Kepler
// kick, CFL time.  The new B never makes a round trip through HBM.
//
// Every corner, face and cell value is computed with the operations of
// ct_core() and prim_cell() (cell_ops.cuh) in the same order, so results are
// bitwise those of the two-kernel form.  Box edges wrap periodically through
// per-axis offset tables, so partial tiles and tiny boxes need no special
// path (halo entries beyond a partial tile are computed and not used).
#pragma once
#include <cuda.h>

#include "cell_ops.cuh"

namespace nmhd {
namespace cell {
namespace epi {

// A box of NI x NJ x NK entries at tile-local origin (OI, OJ, OK) (each 0 or
// -1): local (i, j, k) is the cell (x0 + OI + i, y0 + OJ + j, z0 + OK + k).
// Rows along x are P entries apart, entry i at row position XO + i.
template <int NI_, int NJ_, int NK_, int OI_, int OJ_, int OK_, int P_ = NI_, int XO_ = 0>
struct Box {
  static constexpr int NI = NI_, NJ = NJ_, NK = NK_, OI = OI_, OJ = OJ_, OK = OK_, P = P_, XO = XO_;
  static constexpr int N = P * NJ * NK;  // entries of storage
  static constexpr int DY = P, DZ = P * NJ;
  // index of tile-local cell (a, b, c) in this box
  __device__ static __forceinline__ int at(int a, int b, int c) {
    return ((c - OK) * NJ + (b - OJ)) * P + XO + (a - OI);
  }
};
// A box staged from global memory: rows padded to 16-byte multiples and
// placed so that row position 0 is the 16-byte aligned x0 - 4 (OI = -1) or
// x0 (OI = 0), which lets aligned tiles copy whole rows 16 bytes at a time.
template <int NI, int NJ, int NK, int OI, int OJ, int OK>
using Staged = Box<NI, NJ, NK, OI, OJ, OK, OI == -1 ? 40 : 36, OI == -1 ? 3 : 0>;

// velocities of the stage input: cells x0-1..x0+32, y0-1..y0+4, z0-1..z0+2
using VelBox = Staged<34, 6, 4, -1, -1, -1>;
// B fluxes (flux of a cell = flux through its lower face), with the halo
// their corners read: F_x(B_y), F_y(B_x), F_x(B_z), F_z(B_x), F_y(B_z), F_z(B_y)
using XYF = Staged<33, 6, 2, 0, -1, 0>;
using YXF = Staged<34, 5, 2, -1, 0, 0>;
using XZF = Staged<33, 4, 4, 0, 0, -1>;
using ZXF = Staged<34, 4, 3, -1, 0, 0>;
using YZF = Staged<32, 5, 4, 0, 0, -1>;
using ZYF = Staged<32, 6, 3, 0, -1, 0>;
// corner EMFs (edge of a cell = its lower corner edge): z-edges (XY, YX),
// y-edges (XZ, ZX), x-edges (YZ, ZY)
using ZEdge = Box<33, 5, 2, 0, 0, 0>;
using YEdge = Box<33, 4, 3, 0, 0, 0>;
using XEdge = Box<32, 5, 3, 0, 0, 0>;
// face B of the step's state (staged) and new face B: bx at x0..x0+32, by at
// y0..y0+4, bz at z0..z0+2
using BXs = Staged<33, 4, 2, 0, 0, 0>;
using BYs = Staged<32, 5, 2, 0, 0, 0>;
using BZs = Staged<32, 4, 3, 0, 0, 0>;

// Shared memory of one tile.  The velocity region holds the new face B once
// the corner EMFs are computed; wbf holds the face B of the step's state at
// the same faces.
// Staged and computed boxes in shared memory, each region starting on a
// 128-byte boundary (the tensor-memory-access copies below write whole boxes
// there).
constexpr int r32(int n) { return (n + 31) / 32 * 32; }
constexpr int kXY = 0, kYX = kXY + r32(XYF::N), kXZ = kYX + r32(YXF::N), kZX = kXZ + r32(XZF::N),
              kYZ = kZX + r32(ZXF::N), kZY = kYZ + r32(YZF::N), kBF = kZY + r32(ZYF::N);
constexpr int eXY = 0, eYX = ZEdge::N, eXZ = 2 * ZEdge::N, eZX = eXZ + YEdge::N, eYZ = eZX + YEdge::N,
              eZY = eYZ + XEdge::N, kEdge = r32(eZY + XEdge::N);
constexpr int fBX = 0, fBY = r32(BXs::N), fBZ = fBY + r32(BYs::N), kWB = fBZ + r32(BZs::N);

// Shared memory of one tile.  The velocity region holds the new face B once
// the corner EMFs are computed; wbf holds the face B of the step's state at
// the same faces.
struct __align__(128) Smem {
  float vel[3 * VelBox::N];
  float bf[kBF];
  float edge[kEdge];
  float wbf[kWB];
  int gx[34], gy[6], gz[4];  // wrapped global offsets of x0-1+i, (y0-1+j)*Sx, (z0-1+k)*Sx*Sy
  float red[kThreads / 32];
  unsigned long long mbar;   // completion of the tile's tensor copies
};
static_assert(3 * VelBox::N >= kWB, "face B region");
static_assert((3 * VelBox::N) % 32 == 0 && kBF % 32 == 0 && kEdge % 32 == 0, "128-byte aligned regions");
// bytes the tensor copies of one tile deliver
constexpr unsigned kTileTxBytes =
    4u * (3 * VelBox::N + XYF::N + YXF::N + XZF::N + ZXF::N + YZF::N + ZYF::N + BXs::N + BYs::N + BZs::N);

// Tensor maps (cuTensorMapEncodeTiled, 4-D: x, y, z, field) of the staged
// boxes: per state buffer (0 w0, 1 w1, 2 predictor) the velocity box over
// fields 1-3 and the three face-B boxes; the six B-flux boxes of the flux
// scratch.  `enabled` is 0 where they cannot be made (rows not 16-byte
// multiples); tiles then stage with cp.async.
struct EpiMaps {
  CUtensorMap vel[3], bx[3], by[3], bz[3];
  CUtensorMap xy, yx, xz, zx, yz, zy;
  int enabled;
};

// Global offset of tile-local cell (a, b, c) through the wrapped tables.
__device__ __forceinline__ int goff(const Smem &s, int a, int b, int c) {
  return s.gz[c + 1] + s.gy[b + 1] + s.gx[a + 1];
}

// One 4-byte asynchronous global-to-shared copy (cp.async, sm_80 and later):
// no register holds the value while it is in flight.
__device__ __forceinline__ void cp_async4(unsigned dst, const float *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 16-byte asynchronous copy (both addresses 16-byte aligned), cached in L2 only.
__device__ __forceinline__ void cp_async16(unsigned dst, const float *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

// Tensor copy of box B at tile origin (x0, y0, z0), fields f0.., into shared
// address dst, completing on the tile's mbarrier (cp.async.bulk.tensor; the
// x coordinate x0 + OI - XO is a multiple of 4 floats, 16 bytes).
template <class B>
__device__ __forceinline__ void tma_box(unsigned dst, const CUtensorMap *map, int x0, int y0, int z0, int f0,
                                        unsigned mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x0 + B::OI - B::XO), "r"(y0 + B::OJ), "r"(z0 + B::OK),
      "r"(f0), "r"(mbar)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned mbar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase 0 of the tile's mbarrier: true when the copies
// landed within kTmaWaitTries polls (each poll may itself suspend the thread
// for a while).
constexpr int kTmaWaitTries = 1 << 20;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned mbar) {
  for (int i = 0; i < kTmaWaitTries; ++i)
    if (mbar_try_wait(mbar, 0)) return true;
  return false;
}

// Copy box B of global field src (and, for F > 1 fields, the fields at
// strides of N after it) into shared memory at dst (a shared-space address;
// field f at dst + 4 * f * B::N) with asynchronous copies, so every copy of
// the tile is issued before the first is waited for.
//  vec (rows 16-byte aligned, Sx % 4 == 0): whole padded rows, x0 + OI - XO
//  .. + P - 1, 16 bytes per copy, the tile's threads over all (row, 16-byte
//  chunk) pairs; a chunk that lies beyond an x edge of the box is the chunk
//  Sx away (the periodic wrap moves whole, still aligned, 4-float chunks);
//  otherwise: entry by entry, one row per warp at a time (the row's y and z
//  offsets warp-uniform, a lane's x offsets from the wrapped table).
template <class B, int F>
__device__ __forceinline__ void load_box(const Smem &s, unsigned dst, const float *__restrict__ src, size_t N,
                                         int x0, int nx, bool vec, int tid) {
  if (vec) {
    constexpr int PV = B::P / 4, R = B::NJ * B::NK;
    const int xs = x0 + B::OI - B::XO;
    for (int e = tid; e < R * PV; e += kThreads) {
      const int r = e / PV, v = e - r * PV;
      const int j = r % B::NJ, k = r / B::NJ;
      int xw = xs + 4 * v;  // a multiple of 4 in [-4, Sx + 35]: wrap into [0, Sx)
      if (xw < 0) xw += nx;
      if (xw >= nx) xw %= nx;
      const float *p = src + (s.gz[k + B::OK + 1] + s.gy[j + B::OJ + 1] + xw);
      const unsigned d = dst + 16u * (r * PV + v);
#pragma unroll
      for (int f = 0; f < F; ++f) cp_async16(d + 4u * (f * B::N), p + f * N);
    }
    return;
  }
  const int warp = tid >> 5, lane = tid & 31, i1 = lane + 32;
  const int gx0 = s.gx[lane + B::OI + 1];
  const int gx1 = i1 < B::NI ? s.gx[i1 + B::OI + 1] : 0;
  const unsigned d0 = dst + 4u * (B::XO + lane);
  for (int r = warp; r < B::NJ * B::NK; r += kThreads / 32) {
    const int j = r % B::NJ, k = r / B::NJ;
    const float *row = src + (s.gz[k + B::OK + 1] + s.gy[j + B::OJ + 1]);
    const unsigned d = d0 + 4u * (r * B::P);
#pragma unroll
    for (int f = 0; f < F; ++f) cp_async4(d + 4u * (f * B::N), row + gx0 + f * N);
    if (i1 < B::NI) {
#pragma unroll
      for (int f = 0; f < F; ++f) cp_async4(d + 4u * (f * B::N + 32), row + gx1 + f * N);
    }
  }
}

// Corner EMFs (corner_magnet_flux, mhd_solver.inlrb:641-653) at the edges of
// tile-local cell (a, b, c), with the wind sums in ct_core()'s order: the
// z-edge pair XY (flux F_x(B_y), wind v_y) and YX (F_y(B_x), wind v_x), the
// y-edge pair XZ (F_x(B_z), wind v_z) and ZX (F_z(B_x), wind v_x), the x-edge
// pair YZ (F_y(B_z), wind v_z) and ZY (F_z(B_y), wind v_y).  Neighbour
// entries are at constant offsets from the cell's own.
__device__ __forceinline__ void z_edges(Smem &s, int a, int b, int c) {
  const float *vx = s.vel, *vy = s.vel + VelBox::N;
  const float *xy = s.bf + kXY + XYF::at(a, b, c), *yx = s.bf + kYX + YXF::at(a, b, c);
  const int v = VelBox::at(a, b, c), dx = 1, dy = VelBox::DY;
  const int e = ZEdge::at(a, b, c);
  s.edge[eXY + e] = upwind(vy[v] + vy[v - dy] + vy[v - dx] + vy[v - dx - dy], xy[-XYF::DY], xy[0]);
  s.edge[eYX + e] = upwind(vx[v] + vx[v - dx] + vx[v - dy] + vx[v - dx - dy], yx[-1], yx[0]);
}

__device__ __forceinline__ void y_edges(Smem &s, int a, int j, int c) {
  const float *vx = s.vel, *vz = s.vel + 2 * VelBox::N;
  const float *xz = s.bf + kXZ + XZF::at(a, j, c), *zx = s.bf + kZX + ZXF::at(a, j, c);
  const int v = VelBox::at(a, j, c), dx = 1, dz = VelBox::DZ;
  const int e = YEdge::at(a, j, c);
  s.edge[eXZ + e] = upwind(vz[v] + vz[v - dz] + vz[v - dx] + vz[v - dx - dz], xz[-XZF::DZ], xz[0]);
  s.edge[eZX + e] = upwind(vx[v] + vx[v - dx] + vx[v - dz] + vx[v - dx - dz], zx[-1], zx[0]);
}

__device__ __forceinline__ void x_edges(Smem &s, int i, int b, int c) {
  const float *vy = s.vel + VelBox::N, *vz = s.vel + 2 * VelBox::N;
  const float *yz = s.bf + kYZ + YZF::at(i, b, c), *zy = s.bf + kZY + ZYF::at(i, b, c);
  const int v = VelBox::at(i, b, c), dy = VelBox::DY, dz = VelBox::DZ;
  const int e = XEdge::at(i, b, c);
  s.edge[eYZ + e] = upwind(vz[v] + vz[v - dz] + vz[v - dy] + vz[v - dy - dz], yz[-YZF::DZ], yz[0]);
  s.edge[eZY + e] = upwind(vy[v] + vy[v - dy] + vy[v - dz] + vy[v - dy - dz], zy[-ZYF::DY], zy[0]);
}

// Every corner EMF of the tile: each thread those of its own cell, then the
// upper halo edges (13 rows of 32 and 22 single edges at x0+32).
__device__ __forceinline__ void corner_emfs(Smem &s, int a, int b, int c, int warp, int lane, int tid) {
  z_edges(s, a, b, c);
  y_edges(s, a, b, c);
  x_edges(s, a, b, c);
  for (int r = warp; r < 13; r += kThreads / 32) {
    if (r < 2) z_edges(s, lane, 4, r);
    else if (r < 6) y_edges(s, lane, r - 2, 2);
    else if (r < 9) x_edges(s, lane, 4, r - 6);
    else x_edges(s, lane, r - 9, 2);
  }
  const int k = tid - (kThreads - 32);
  if (k >= 0 && k < 10) z_edges(s, 32, k % 5, k / 5);
  else if (k >= 10 && k < 22) y_edges(s, 32, (k - 10) % 4, (k - 10) / 4);
}

// New face B (ct_core()'s face sums) of the lower x-, y- or z-face of
// tile-local cell (a, b, c), from the corner EMFs and the face's B at the
// start of the step (wbf: that component's field at the face).
template <bool kPow2>
__device__ __forceinline__ float new_bx(const Smem &s, const GridParams &g, float wbf, int a, int j, int c, float dt) {
  const float *E = s.edge;
  const int z = ZEdge::at(a, j, c), y = YEdge::at(a, j, c);
  const float XY00 = E[eXY + z], XY01 = E[eXY + z + ZEdge::DY];
  const float XZ00 = E[eXZ + y], XZ01 = E[eXZ + y + YEdge::DZ];
  const float YX00 = E[eYX + z], YX01 = E[eYX + z + ZEdge::DY];
  const float ZX00 = E[eZX + y], ZX01 = E[eZX + y + YEdge::DZ];
  float pb = 0.0f;
  pb = pb + 0.5f * (divs<kPow2>(XY01 - XY00, g.dy, g.inv_dy) + divs<kPow2>(XZ01 - XZ00, g.dz, g.inv_dz));
  pb = pb - divs<kPow2>(0.5f * (YX01 - YX00), g.dy, g.inv_dy);
  pb = pb - divs<kPow2>(0.5f * (ZX01 - ZX00), g.dz, g.inv_dz);
  return wbf + dt * pb;
}

template <bool kPow2>
__device__ __forceinline__ float new_by(const Smem &s, const GridParams &g, float wbf, int i, int b, int c, float dt) {
  const float *E = s.edge;
  const int z = ZEdge::at(i, b, c), x = XEdge::at(i, b, c);
  const float XY00 = E[eXY + z], XY10 = E[eXY + z + 1];
  const float YZ00 = E[eYZ + x], YZ01 = E[eYZ + x + XEdge::DZ];
  const float YX00 = E[eYX + z], YX10 = E[eYX + z + 1];
  const float ZY00 = E[eZY + x], ZY01 = E[eZY + x + XEdge::DZ];
  float pb = 0.0f;
  pb = pb - divs<kPow2>(0.5f * (XY10 - XY00), g.dx, g.inv_dx);
  pb = pb + 0.5f * (divs<kPow2>(YZ01 - YZ00, g.dz, g.inv_dz) + divs<kPow2>(YX10 - YX00, g.dx, g.inv_dx));
  pb = pb - divs<kPow2>(0.5f * (ZY01 - ZY00), g.dz, g.inv_dz);
  return wbf + dt * pb;
}

template <bool kPow2>
__device__ __forceinline__ float new_bz(const Smem &s, const GridParams &g, float wbf, int i, int j, int c, float dt) {
  const float *E = s.edge;
  const int y = YEdge::at(i, j, c), x = XEdge::at(i, j, c);
  const float XZ00 = E[eXZ + y], XZ10 = E[eXZ + y + 1];
  const float YZ00 = E[eYZ + x], YZ10 = E[eYZ + x + XEdge::DY];
  const float ZX00 = E[eZX + y], ZX10 = E[eZX + y + 1];
  const float ZY00 = E[eZY + x], ZY10 = E[eZY + x + XEdge::DY];
  float pb = 0.0f;
  pb = pb - divs<kPow2>(0.5f * (XZ10 - XZ00), g.dx, g.inv_dx);
  pb = pb - divs<kPow2>(0.5f * (YZ10 - YZ00), g.dy, g.inv_dy);
  pb = pb + 0.5f * (divs<kPow2>(ZX10 - ZX00, g.dx, g.inv_dx) + divs<kPow2>(ZY10 - ZY00, g.dy, g.inv_dy));
  return wbf + dt * pb;
}

// New face B of the tile's faces (each thread its cell's three) and of the
// upper halo faces (by at y0+4 and bz at z0+2 as 6 rows of 32, bx at x0+32
// as 8 single faces), into the shared face region.
template <bool kPow2>
__device__ __forceinline__ void face_b(Smem &s, const GridParams &g, int a, int b, int c, int warp, int lane,
                                       float dt) {
  float *F = s.vel;  // the velocities are dead once the corner EMFs exist
  const float *W = s.wbf;
  float hb = 0.0f;
  int hr = -1;
  if (warp < 2) {
    hr = fBY + BYs::at(lane, 4, warp);
    hb = new_by<kPow2>(s, g, W[hr], lane, 4, warp, dt);
  } else if (warp < 6) {
    hr = fBZ + BZs::at(lane, warp - 2, 2);
    hb = new_bz<kPow2>(s, g, W[hr], lane, warp - 2, 2, dt);
  } else if (warp == 6 && lane < 8) {
    hr = fBX + BXs::at(32, lane & 3, lane >> 2);
    hb = new_bx<kPow2>(s, g, W[hr], 32, lane & 3, lane >> 2, dt);
  }
  const int ix = fBX + BXs::at(a, b, c), iy = fBY + BYs::at(a, b, c), iz = fBZ + BZs::at(a, b, c);
  F[ix] = new_bx<kPow2>(s, g, W[ix], a, b, c, dt);
  F[iy] = new_by<kPow2>(s, g, W[iy], a, b, c, dt);
  F[iz] = new_bz<kPow2>(s, g, W[iz], a, b, c, dt);
  if (hr >= 0) F[hr] = hb;
}

// The rest of the stage for tile-local cell (a, b, c) at global (x, y, z),
// offset o: prim_cell() with the new face B taken from shared memory, and the
// new B of the cell's lower faces written with the other fields.
template <bool kPow2>
__device__ __forceinline__ float finish_cell(const Smem &s, const GridParams &g, const float *__restrict__ wb,
                                             float *__restrict__ wo, const float *__restrict__ flux, int a, int b,
                                             int c, int x, int y, int z, float dt, bool final_stage, int *bad) {
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const int xp = x + 1 < g.sx ? 1 : 1 - g.sx;
  const int yp = (y + 1 < g.sy ? 1 : 1 - g.sy) * g.sx;
  const int zp = (z + 1 < g.sz ? 1 : 1 - g.sz) * g.sx * g.sy;
  const float *Fx = flux, *Fy = flux + 7 * N, *Fz = flux + 14 * N;
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
  const float *W = s.wbf;
  const float bxl = W[fBX + BXs::at(a, b, c)], bxh = W[fBX + BXs::at(a + 1, b, c)];
  const float byl = W[fBY + BYs::at(a, b, c)], byh = W[fBY + BYs::at(a, b + 1, c)];
  const float bzl = W[fBZ + BZs::at(a, b, c)], bzh = W[fBZ + BZs::at(a, b, c + 1)];
  const float mx0 = rho0 * vx0, my0 = rho0 * vy0, mz0 = rho0 * vz0;
  const float e0 = p0 / gm1 + 0.5f * rho0 * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0) +
                   0.25f * (bxl * bxl + bxh * bxh + byl * byl + byh * byh + bzl * bzl + bzh * bzh);
  const float rho = rho0 + dt * pace[0];
  const float mx = mx0 + dt * pace[1];
  const float my = my0 + dt * pace[2];
  const float mz = mz0 + dt * pace[3];
  const float ene = e0 + dt * pace[4];
  const float *Fb = s.vel;
  const float bx0 = Fb[fBX + BXs::at(a, b, c)], bx1 = Fb[fBX + BXs::at(a + 1, b, c)];
  const float by0 = Fb[fBY + BYs::at(a, b, c)], by1 = Fb[fBY + BYs::at(a, b + 1, c)];
  const float bz0 = Fb[fBZ + BZs::at(a, b, c)], bz1 = Fb[fBZ + BZs::at(a, b, c + 1)];
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
  wo[5 * N + o] = bx0;
  wo[6 * N + o] = by0;
  wo[7 * N + o] = bz0;
  float tcfl = __uint_as_float(0x7f800000u);
  if (final_stage) {
    *bad = !(rho > 0.0f) || !(po > 0.0f) || !isfinite(vxo) || !isfinite(vyo) || !isfinite(vzo) ||
           !isfinite(bx0) || !isfinite(by0) || !isfinite(bz0);
    const bool margin_cell = (y < g.my) || (y >= g.sy - g.my) || (g.mz > 0 && (z < g.mz || z >= g.sz - g.mz - 1));
    if (!margin_cell) {
      const float b2 = fmaxf(bx0 * bx0, bx1 * bx1) + fmaxf(by0 * by0, by1 * by1) + fmaxf(bz0 * bz0, bz1 * bz1);
      const float cs = sqrtf((g.gamma * po + b2) / rho);
      tcfl = fminf(fminf(g.cfl * g.dx / fabsf(vxo + cs), g.cfl * g.dy / fabsf(vyo + cs)),
                   g.cfl * g.dz / fabsf(vzo + cs));
    }
  }
  return tcfl;
}

// The whole epilogue of one tile at (x0, y0, z0); every thread of the CTA
// calls it.  maps: the tensor maps of these buffers (interior tiles stage by
// tensor copies), or NULL (every tile stages with cp.async).  win: stage
// input (velocities), wb: state at the start of the step, wo: stage output.
// Returns the thread's CFL time (inf if none).
template <bool kPow2>
__device__ __forceinline__ float tile_epilogue(Smem &s, const GridParams &g, const EpiMaps *maps, int in_buf,
                                               int base_buf, const float *__restrict__ win,
                                               const float *__restrict__ wb, float *__restrict__ wo,
                                               const float *__restrict__ flux, int x0, int y0, int z0, float dt,
                                               bool final_stage, int *bad, int *timed_out) {
  // the thread's cell (a, b, c) of the tile, from its linear index: the same
  // for a 32 x 4 x 2 block (the single-box kernel) and a 1-D block of 256
  // threads (the batched kernel)
  const int tid = (threadIdx.z * BY + threadIdx.y) * BX + threadIdx.x;
  const int a = tid % BX, b = tid / BX % BY, c = tid / (BX * BY);
  const size_t N = (size_t)g.n;
  {
    // L2 prefetch of the lines the cell update reads later: each warp holds
    // one x row of 32 cells (one 128-byte line per field), lanes 0-14 take
    // the 15 mass/momentum/energy face-flux fields, lanes 15-22 the 8 fields
    // of the step's state
    const int lane = tid & 31, y = y0 + b, z = z0 + c;
    if (lane < 23 && y < g.sy && z < g.sz) {
      const size_t o = (size_t)(z * g.sy + y) * g.sx + x0;
      const float *p = lane < 15 ? flux + (size_t)(lane / 5 * 7 + lane % 5) * N + o : wb + (size_t)(lane - 15) * N + o;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }
  const unsigned vs = (unsigned)__cvta_generic_to_shared(s.vel), bs = (unsigned)__cvta_generic_to_shared(s.bf),
                 ws = (unsigned)__cvta_generic_to_shared(s.wbf),
                 mb = (unsigned)__cvta_generic_to_shared(&s.mbar);
  // Tiles whose staged boxes (x0-4..x0+35, y0-1..y0+4, z0-1..z0+2) lie inside
  // the box need no periodic wrap: one thread stages all of them with ten
  // tensor copies.  The others stage entry by entry through the wrapped
  // offset tables (16-byte row chunks when only y or z wraps).
  const bool tma = maps && maps->enabled && x0 >= 4 && x0 + 36 <= g.sx && y0 >= 1 && y0 + 5 <= g.sy && z0 >= 1 &&
                   z0 + 3 <= g.sz;
  if (tma) {
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(kTileTxBytes)
                   : "memory");
      tma_box<VelBox>(vs, &maps->vel[in_buf], x0, y0, z0, 1, mb);
      tma_box<XYF>(bs + 4 * kXY, &maps->xy, x0, y0, z0, 5, mb);
      tma_box<YXF>(bs + 4 * kYX, &maps->yx, x0, y0, z0, 13, mb);
      tma_box<XZF>(bs + 4 * kXZ, &maps->xz, x0, y0, z0, 6, mb);
      tma_box<ZXF>(bs + 4 * kZX, &maps->zx, x0, y0, z0, 19, mb);
      tma_box<YZF>(bs + 4 * kYZ, &maps->yz, x0, y0, z0, 12, mb);
      tma_box<ZYF>(bs + 4 * kZY, &maps->zy, x0, y0, z0, 20, mb);
      tma_box<BXs>(ws + 4 * fBX, &maps->bx[base_buf], x0, y0, z0, 5, mb);
      tma_box<BYs>(ws + 4 * fBY, &maps->by[base_buf], x0, y0, z0, 6, mb);
      tma_box<BZs>(ws + 4 * fBZ, &maps->bz[base_buf], x0, y0, z0, 7, mb);
    }
  } else {
    if (tid < 34) s.gx[tid] = wrap_any(x0 - 1 + tid, g.sx);
    else if (tid < 40) s.gy[tid - 34] = wrap_any(y0 - 1 + (tid - 34), g.sy) * g.sx;
    else if (tid < 44) s.gz[tid - 40] = wrap_any(z0 - 1 + (tid - 40), g.sz) * g.sx * g.sy;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  if (tma) {
    // every thread waits for the copies (bounded); the outcome is made
    // uniform over the CTA
    const bool ok = __syncthreads_and(mbar_wait_bounded(mb));
    if (!ok) {
      // the copies did not land in time: flag it and wait once more (bounded)
      // so that none is still writing when the CTA exits
      *timed_out = 1;
      mbar_wait_bounded(mb);
      __syncthreads();
      if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
      return __uint_as_float(0x7f800000u);
    }
    // every thread has passed the wait: the barrier's word is released
    if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
  } else {
    // whole 16-byte row chunks where rows are 16-byte aligned
    const bool vec = (g.sx & 3) == 0;
    load_box<VelBox, 3>(s, vs, win + N, N, x0, g.sx, vec, tid);
    load_box<XYF, 1>(s, bs + 4 * kXY, flux + 5 * N, N, x0, g.sx, vec, tid);
    load_box<YXF, 1>(s, bs + 4 * kYX, flux + 13 * N, N, x0, g.sx, vec, tid);
    load_box<XZF, 1>(s, bs + 4 * kXZ, flux + 6 * N, N, x0, g.sx, vec, tid);
    load_box<ZXF, 1>(s, bs + 4 * kZX, flux + 19 * N, N, x0, g.sx, vec, tid);
    load_box<YZF, 1>(s, bs + 4 * kYZ, flux + 12 * N, N, x0, g.sx, vec, tid);
    load_box<ZYF, 1>(s, bs + 4 * kZY, flux + 20 * N, N, x0, g.sx, vec, tid);
    load_box<BXs, 1>(s, ws + 4 * fBX, wb + 5 * N, N, x0, g.sx, vec, tid);
    load_box<BYs, 1>(s, ws + 4 * fBY, wb + 6 * N, N, x0, g.sx, vec, tid);
    load_box<BZs, 1>(s, ws + 4 * fBZ, wb + 7 * N, N, x0, g.sx, vec, tid);
    cp_async_wait_all();
    __syncthreads();
  }
  corner_emfs(s, a, b, c, warp, lane, tid);
  __syncthreads();
  face_b<kPow2>(s, g, a, b, c, warp, lane, dt);
  __syncthreads();
  const int x = x0 + a, y = y0 + b, z = z0 + c;
  if (x < g.sx && y < g.sy && z < g.sz)
    return finish_cell<kPow2>(s, g, wb, wo, flux, a, b, c, x, y, z, dt, final_stage, bad);
  return __uint_as_float(0x7f800000u);
}

}  // namespace epi
}  // namespace cell
}  // namespace nmhd
