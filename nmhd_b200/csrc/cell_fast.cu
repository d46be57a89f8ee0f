// Fast-arithmetic flux kernel (NMHD_FLAG_FAST_ARITHMETIC), sm_100a.
//
// The same staging and reconstruction + HLLD per face as k_cell_flux_staged
// (cell_stage.cu, cell_flux_staged.cuh), but this translation unit is
// compiled with multiply-add contraction and
// approximate division and square root, and the reference's FP64
// sub-expressions of the HLLD solver are evaluated in float (NMHD_FAST_ARITH in
// mhd_math.cuh).  The update kernels stay the exact ones.  The face fluxes then
// differ from the reference's by rounding-size amounts: the state after one
// step is within 1e-5 (relative to each quantity's scale) of the reference's,
// not bitwise equal to it.
#define NMHD_FAST_ARITH 1
#include "cell_flux_staged.cuh"

namespace nmhd {
namespace {

using namespace cell;

__global__ void __launch_bounds__(kThreads, 4)
    k_cell_flux_fast(const __grid_constant__ sfx::FluxMaps maps, GridParams g, StepCtl *ctl, const float *w0,
                     const float *w1, const float *wp, float *__restrict__ flux, int in_sel, int half) {
  __shared__ sfx::Smem s;
  if (ctl->done) return;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const int tid = (threadIdx.z * BY + threadIdx.y) * BX + threadIdx.x;
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY, z0 = blockIdx.z * BZ;
  if (!sfx::stage(s, g, &maps, pick_index(ctl, in_sel), pick(ctl, in_sel, w0, w1, wp), x0, y0, z0, tid)) {
    if (tid == 0) atomicOr(&ctl->status, kStatusTimeout);
    return;
  }
  const int x = x0 + threadIdx.x, y = y0 + threadIdx.y, z = z0 + threadIdx.z;
  if (x < g.sx && y < g.sy && z < g.sz)
    sfx::flux_cell_staged(g, s, flux, threadIdx.x, threadIdx.y, threadIdx.z, x, y, z, dt);
}

}  // namespace

void launch_cell_flux_fast(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                           int in_sel, int half, const EpilogueMaps *maps, cudaStream_t st) {
  static const EpilogueMaps kNone = {};  // enabled = 0: cp.async staging only
  const dim3 grid((g.sx + BX - 1) / BX, (g.sy + BY - 1) / BY, (g.sz + BZ - 1) / BZ);
  k_cell_flux_fast<<<grid, dim3(BX, BY, BZ), 0, st>>>(maps ? maps->f : kNone.f, g, ctl, w0, w1, wp, flux, in_sel,
                                                       half);
}

}  // namespace nmhd
