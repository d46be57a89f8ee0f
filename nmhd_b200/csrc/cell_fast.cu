// Fast-arithmetic flux kernel (NMHD_FLAG_FAST_ARITHMETIC), sm_100a.
//
// The same reconstruction + HLLD per face as k_cell_flux (cell_stage.cu), but
// this translation unit is compiled with multiply-add contraction and
// approximate division and square root, and the reference's FP64
// sub-expressions of the HLLD solver are evaluated in float (NMHD_FAST_ARITH in
// mhd_math.cuh).  The update kernels stay the exact ones.  The face fluxes then
// differ from the reference's by rounding-size amounts: the state after one
// step is within 1e-5 (relative to each quantity's scale) of the reference's,
// not bitwise equal to it.
#define NMHD_FAST_ARITH 1
#include "cell_ops.cuh"

namespace nmhd {
namespace {

using namespace cell;

__global__ void __launch_bounds__(kThreads, 4) k_cell_flux_fast(GridParams g, const StepCtl *ctl, const float *w0,
                                                                const float *w1, const float *wp,
                                                                float *__restrict__ flux, int in_sel, int half) {
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = blockIdx.z * BZ + threadIdx.z;
  if (x >= g.sx || y >= g.sy || z >= g.sz) return;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  flux_cell(g, pick(ctl, in_sel, w0, w1, wp), flux, x, y, z, dt);
}

}  // namespace

void launch_cell_flux_fast(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                           int in_sel, int half, cudaStream_t st) {
  const dim3 grid((g.sx + BX - 1) / BX, (g.sy + BY - 1) / BY, (g.sz + BZ - 1) / BZ);
  k_cell_flux_fast<<<grid, dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, half);
}

}  // namespace nmhd
