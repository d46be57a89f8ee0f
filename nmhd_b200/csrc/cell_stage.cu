// Per-cell stage kernels (variant 2, the default) of the B200 ideal-MHD time
// step, sm_100a: one thread per cell on 32 x 4 x 2 CTAs.
//
//  k_cell_flux  reconstruction + HLLD on the cell's lower x-, y- and z-face
//               (calc_flux_kernel<X,Y,Z>, src/library/mhd_solver.inlrb:562-636);
//               21 flux values per cell go to scratch.
//  k_cell_ct    corner EMFs and the face-B update (:641-714), written into the
//               output state.
//  k_cell_prim  flux divergence (add_flux_kernel :689-693), conserved update
//               (:762-835), primitive recovery (:779-795), the Kepler kick
//               (:837-848), and in the final stage the CFL reduction and clock
//               update (:496-521, 870-901, 981).
// The per-cell work lives in cell_ops.cuh, shared with the batch kernels.
#include "cell_ops.cuh"

namespace nmhd {

namespace {

using namespace cell;

__global__ void __launch_bounds__(kThreads, 3) k_cell_flux(GridParams g, const StepCtl *ctl, const float *w0,
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

template <bool kPow2>
__global__ void __launch_bounds__(kThreads, 4) k_cell_ct(GridParams g, const StepCtl *ctl, float *w0,
                                                         float *w1, float *wp,
                                                         const float *__restrict__ flux, int in_sel,
                                                         int out_sel, int half) {
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = blockIdx.z * BZ + threadIdx.z;
  if (x >= g.sx || y >= g.sy || z >= g.sz) return;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  ct_cell<kPow2>(g, pick(ctl, in_sel, w0, w1, wp), pick(ctl, 0, w0, w1, wp),
                 const_cast<float *>(pick(ctl, out_sel, w0, w1, wp)), flux, x, y, z, dt);
}

template <bool kPow2>
__global__ void __launch_bounds__(kThreads, 3) k_cell_prim(GridParams g, StepCtl *ctl, float *w0,
                                                           float *w1, float *wp,
                                                           const float *__restrict__ flux, float *dt_hist,
                                                           int out_sel, int half, int final_stage) {
  __shared__ float red[kThreads / 32];
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = blockIdx.z * BZ + threadIdx.z;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  float tcfl = __uint_as_float(0x7f800000u);
  int bad = 0;
  if (x < g.sx && y < g.sy && z < g.sz)
    tcfl = prim_cell<kPow2>(g, pick(ctl, 0, w0, w1, wp), const_cast<float *>(pick(ctl, out_sel, w0, w1, wp)),
                            flux, x, y, z, dt, final_stage != 0, &bad);
  if (final_stage) finish_tile(ctl, gridDim.x * gridDim.y * gridDim.z, tcfl, bad, dt_hist, red);
}

dim3 cell_grid(const GridParams &g) {
  return dim3((g.sx + BX - 1) / BX, (g.sy + BY - 1) / BY, (g.sz + BZ - 1) / BZ);
}

}  // namespace

void launch_cell_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                      int in_sel, int half, cudaStream_t st) {
  k_cell_flux<<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, half);
}

void launch_cell_update(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                        float *dt_hist, int in_sel, int out_sel, int half, int final_stage, cudaStream_t st) {
  if (g.pow2_spacing) {
    k_cell_ct<true><<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, out_sel, half);
    k_cell_prim<true><<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, dt_hist, out_sel,
                                                               half, final_stage);
  } else {
    k_cell_ct<false><<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, out_sel, half);
    k_cell_prim<false><<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, dt_hist, out_sel,
                                                                half, final_stage);
  }
}

}  // namespace nmhd
