// Face fluxes of a 32 x 4 x 2-cell tile from a shared-memory copy of the
// stage input (kernel variant 5's flux kernel).
//
// The per-cell flux kernel reads its 40-odd stencil values per face from
// global memory, and each read costs a 64-bit address computed from the
// cell's wrapped neighbour offsets: on the 128x256x64 shearing box a fifth of
// its instructions are integer address arithmetic.  Here the tile first
// copies all 8 fields of the cells x0-2..x0+32, y0-2..y0+4, z0-2..z0+2 (the
// union of the three axes' 4-cell stencils and the +1 transverse neighbours
// of the face-centred B) into shared memory, with one tensor copy for tiles
// away from the box edges; every stencil read is then a shared load at a
// constant or axis-stride offset.  The arithmetic is face_flux()'s, the same
// code the per-cell kernel runs, so the fluxes are bitwise the same.
#pragma once
#include "cell_epilogue.cuh"

namespace nmhd {
namespace cell {
namespace sfx {

// Staged box: rows of P = 40 floats starting at the 16-byte aligned x0 - 4
// (x0 at row position 4), NJ = 7 rows (y0-2..y0+4) per plane, NK = 5 planes
// (z0-2..z0+2), the 8 fields FS floats apart.
constexpr int P = 40, NJ = 7, NK = 5, XO = 4;
constexpr int DY = P, DZ = P * NJ, FS = P * NJ * NK;
constexpr unsigned kTxBytes = 4u * 8u * FS;

struct __align__(128) Smem {
  float w[8 * FS];
  int gx[P], gy[NJ], gz[NK];  // wrapped global offsets of x0-4+i, (y0-2+j)*Sx, (z0-2+k)*Sx*Sy
  unsigned long long mbar;
};

// Tensor maps (4-D: x, y, z, field) of the staged box over each state buffer
// (0 w0, 1 w1, 2 predictor); `enabled` 0 where they cannot be made.
struct FluxMaps {
  CUtensorMap w[3];
  int enabled;
};

// Shared index of tile-local cell (a, b, c).
__device__ __forceinline__ int at(int a, int b, int c) { return ((c + 2) * NJ + (b + 2)) * P + XO + a; }

// Copies the stage input w around tile (x0, y0, z0) into s.w.  Tiles whose box
// lies inside the grid: one tensor copy issued by thread 0, completing on the
// mbarrier (bounded wait; false if it timed out).  Others: cp.async through
// the wrapped offset tables, 16-byte row chunks where Sx % 4 == 0, else entry
// by entry.  Every thread of the CTA calls it.
__device__ __forceinline__ bool stage(Smem &s, const GridParams &g, const FluxMaps *maps, int buf,
                                      const float *__restrict__ w, int x0, int y0, int z0, int tid) {
  const size_t N = (size_t)g.n;
  const unsigned ds = (unsigned)__cvta_generic_to_shared(s.w), mb = (unsigned)__cvta_generic_to_shared(&s.mbar);
  const bool tma = maps && maps->enabled && x0 >= 4 && x0 + 36 <= g.sx && y0 >= 2 && y0 + 5 <= g.sy && z0 >= 2 &&
                   z0 + 3 <= g.sz;
  if (tma) {
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(kTxBytes) : "memory");
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
          "%4, %5}], [%6];" ::"r"(ds),
          "l"(reinterpret_cast<unsigned long long>(&maps->w[buf])), "r"(x0 - XO), "r"(y0 - 2), "r"(z0 - 2), "r"(0),
          "r"(mb)
          : "memory");
    }
    __syncthreads();
    const bool ok = __syncthreads_and(epi::mbar_wait_bounded(mb));
    if (!ok) {
      // flag it and wait once more (bounded) so that no copy is still
      // writing when the CTA exits
      epi::mbar_wait_bounded(mb);
      __syncthreads();
      if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
      return false;
    }
    if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mb) : "memory");
    return true;
  }
  if (tid < P) s.gx[tid] = wrap_any(x0 - XO + tid, g.sx);
  else if (tid < P + NJ) s.gy[tid - P] = wrap_any(y0 - 2 + (tid - P), g.sy) * g.sx;
  else if (tid < P + NJ + NK) s.gz[tid - P - NJ] = wrap_any(z0 - 2 + (tid - P - NJ), g.sz) * g.sx * g.sy;
  __syncthreads();
  constexpr int R = NJ * NK;
  if ((g.sx & 3) == 0) {
    // 16-byte chunks of the rows; a chunk beyond an x edge of the box is the
    // (aligned) chunk Sx away
    constexpr int PV = P / 4;
    const int xs = x0 - XO;
    for (int e = tid; e < R * PV; e += kThreads) {
      const int r = e / PV, v = e - r * PV;
      int xw = xs + 4 * v;  // a multiple of 4 in [-4, Sx + 35]: wrap into [0, Sx)
      if (xw < 0) xw += g.sx;
      if (xw >= g.sx) xw %= g.sx;
      const float *src = w + (s.gz[r / NJ] + s.gy[r % NJ] + xw);
      const unsigned d = ds + 16u * (r * PV + v);
#pragma unroll
      for (int f = 0; f < 8; ++f) epi::cp_async16(d + 4u * (f * FS), src + f * N);
    }
  } else {
    // one row per warp at a time: lanes 0-31 and 0-7 again for entries 32-39
    const int warp = tid >> 5, lane = tid & 31;
    const int gx0 = s.gx[lane], gx1 = lane < P - 32 ? s.gx[lane + 32] : 0;
    for (int r = warp; r < R; r += kThreads / 32) {
      const float *row = w + (s.gz[r / NJ] + s.gy[r % NJ]);
      const unsigned d = ds + 4u * (r * P + lane);
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        epi::cp_async4(d + 4u * (f * FS), row + gx0 + f * N);
        if (lane < P - 32) epi::cp_async4(d + 4u * (f * FS + 32), row + gx1 + f * N);
      }
    }
  }
  epi::cp_async_wait_all();
  __syncthreads();
  return true;
}

// The three lower-face fluxes of tile-local cell (a, b, c) at global (x, y,
// z), from the staged copy: flux_cell() with shared addressing.
__device__ __forceinline__ void flux_cell_staged(const GridParams &g, const Smem &s, float *__restrict__ flux,
                                                 int a, int b, int c, int x, int y, int z, float dt) {
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const int ci = at(a, b, c);
#pragma unroll 1
  for (int ax = 0; ax < 3; ++ax) {
    const int sa = ax == 0 ? 1 : ax == 1 ? DY : DZ;
    const int t1 = ax == 0 ? DY : ax == 1 ? DZ : 1;
    const int t2 = ax == 0 ? DZ : ax == 1 ? 1 : DY;
    face_flux<SharedLd, int>(g, s.w, FS, ci, ax, -2 * sa, -sa, sa, t1, t2, y, dt, flux, N, o);
  }
}

}  // namespace sfx
}  // namespace cell

// The tensor maps of one solver's buffers (make_epilogue_maps): the fused
// epilogue's and the staged flux kernels'.
struct EpilogueMaps {
  cell::epi::EpiMaps m;
  cell::sfx::FluxMaps f;
};

}  // namespace nmhd
