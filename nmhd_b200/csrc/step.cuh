// Internal interface between the C ABI (solver.cu) and the step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/nmhd.h"

namespace nmhd {

// Runtime constants of one box (the reference's simulation_config.h values).
struct GridParams {
  int sx, sy, sz;  // cells including margins
  int n;           // sx*sy*sz
  int my, mz;      // margins
  float dx, dy, dz;
  float gamma, cfl;
  float q, omega;
  float corner_y;  // origin of the Kepler radial coordinate (-kExtentY/2)
  float extent_x;  // kExtentX
  double rel_vel;  // relative_velocity(): -q*Omega*kLocalExtentY
  int shear;       // shearing box: Kepler acceleration + shearing-periodic Y margins
  int order2;      // minbee (2) vs piecewise-constant (1) reconstruction
  // 1/dx, 1/dy, 1/dz; when all three spacings are powers of two (pow2_spacing),
  // x / d == x * (1/d) exactly and kernels may multiply instead of divide.
  float inv_dx, inv_dy, inv_dz;
  int pow2_spacing;
};

// Device-resident step control.  The time step is a pure function of
// (cfl_cur, time, goal), evaluated identically by every block that needs it, so
// no host round trip is needed between steps.
struct StepCtl {
  double time;                // current_time (FP64, as the reference's PreciseReal)
  long long generation;
  unsigned cfl_cur;           // float bits: min over cells of the CFL time (this step)
  unsigned cfl_next;          // accumulated by the final stage for the next step
  float goal;                 // goal_time as float (the reference's `Real goal_time`)
  int parity;                 // which of the two state buffers holds the current state
  int done;                   // goal reached or run stopped: later kernels return at once
  int status;                 // kStatus* bits
  unsigned blocks_done;       // last-block detection in the final stage
  int hist_cap;
  // Frozen time steps (adjoint and its finite-difference checks): when dt_seq
  // is set, step n uses dt_seq[generation - dt_seq_base] instead of the CFL dt.
  const float *dt_seq;
  long long dt_seq_base;
};

// kStatusTimeout: a bounded wait inside a kernel (for its tensor copies) gave
// up; the kernel stopped without writing its results.
enum : int { kStatusNumerical = 1, kStatusBadDt = 2, kStatusTimeout = 4 };

// Box constants from a configuration, with the reference's float chains.
GridParams derive_grid(const nmhd_config &c);
// The runtime configuration's rules (nmhd_create's checks, shared by every
// entry point that takes an nmhd_config): NMHD_OK, or a status and `why`.
nmhd_status validate_config(const nmhd_config *c, std::string &why);
constexpr int kDtHistCap = 4096;
constexpr int kFluxFields = 21;  // 3 face directions x 7 flux components

// Launchers (all asynchronous on `stream`).
void launch_cfl_all(const GridParams &g, StepCtl *ctl, float *w0, float *w1, cudaStream_t stream);
void launch_cfl_margin(const GridParams &g, StepCtl *ctl, float *w0, float *w1, cudaStream_t stream);
void launch_fill(const GridParams &g, StepCtl *ctl, float *w0, float *w1, cudaStream_t stream);
// Margins of the RK2 predictor wp refilled at t + dt/2 (NMHD_FLAG_HALO_PER_STAGE).
void launch_fill_predictor(const GridParams &g, StepCtl *ctl, float *wp, cudaStream_t stream);
// Radial slab halo: gather the outgoing Y-boundary messages / scatter the
// incoming ones into the Y margins and copy the Z margins.
void launch_halo_pack(const GridParams &g, StepCtl *ctl, const float *w0, const float *w1, float *send_inc,
                      float *send_dec, cudaStream_t stream);
void launch_halo_unpack(const GridParams &g, StepCtl *ctl, float *w0, float *w1, const float *recv_inc,
                        const float *recv_dec, cudaStream_t stream);
// CFL-time slots (StepCtl::cfl_cur as float) of the slabs of one process.
constexpr int kMaxSlots = 64;
struct CflSlots {
  float *p[kMaxSlots];
  int n;
};
void launch_cfl_min(const CflSlots &slots, cudaStream_t stream);
// One RK stage: fluxes from buffer `in_sel`, conserved state from the current
// buffer, result into `out_sel` (0 current, 1 next, 2 predictor); `half`
// selects dt/2; `final_stage` reduces the next CFL time and advances the clock.
void launch_stage(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                  float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                  cudaStream_t stream);
// The two kernels of a stage, separately (for per-kernel timing).
void launch_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                 int in_sel, int half, cudaStream_t stream);
void launch_update(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                   float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                   cudaStream_t stream);
// Tile shape of the tiled stage kernels: rows per CTA (4, 8 or 16; the CTA
// is 32 x ty threads) and z planes per CTA (0: the whole box height).
struct TileShape {
  int ty;
  int zc;
};
// One RK stage with the tiled kernels (k_tile_flux + k_tile_ct); unew holds
// 5 and bflux 6 fields of Sx*Sy*Sz floats.
void launch_tile_stage(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew,
                       float *bflux, float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                       const TileShape &shape, cudaStream_t stream);
// The staged flux kernel with fast arithmetic (NMHD_FLAG_FAST_ARITHMETIC,
// cell_fast.cu); `maps` as for launch_cell_flux_staged.
struct EpilogueMaps;
void launch_cell_flux_fast(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                           int in_sel, int half, const EpilogueMaps *maps, cudaStream_t stream);
// Per-cell stage kernels with 32x4x2 CTAs (flux: 21 fields of scratch).
void launch_cell_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                      int in_sel, int half, cudaStream_t stream);
void launch_cell_update(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                        float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                        cudaStream_t stream);
// The update of a stage in one kernel (variant 4): constrained transport and
// conserved update fused, corner EMFs and new face B in shared memory.
// `maps` (make_epilogue_maps, for these w0, w1, wp and flux buffers) lets
// interior tiles stage their inputs with tensor copies; NULL: cp.async only.
struct EpilogueMaps;
EpilogueMaps *make_epilogue_maps(const GridParams &g, float *w0, float *w1, float *wp, float *flux);
void free_epilogue_maps(EpilogueMaps *m);
void launch_cell_update_fused(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                              float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                              const EpilogueMaps *maps, cudaStream_t stream);
// The face fluxes of a stage from a shared-memory copy of each tile's
// stencil (variant 5), the same fluxes as launch_cell_flux; `maps` as above
// (interior tiles copy with one tensor copy).
void launch_cell_flux_staged(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                             int in_sel, int half, const EpilogueMaps *maps, cudaStream_t stream);
// One RK stage with the per-cell kernels as a pipeline over chunks of z_chunk
// planes (variant 3), so each chunk's face fluxes are consumed from L2.
void launch_cell_stage_chunked(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                               float *dt_hist, int in_sel, int out_sel, int half, int final_stage, int z_chunk,
                               cudaStream_t stream);
// The two kernels of a tiled stage, separately (for per-kernel timing).
void launch_tile_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew,
                      float *bflux, int in_sel, int half, const TileShape &shape, cudaStream_t stream);
void launch_tile_ct(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew,
                    float *bflux, float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                    const TileShape &shape, cudaStream_t stream);
void launch_diag(const GridParams &g, StepCtl *ctl, float *w0, float *w1, double *acc,
                 cudaStream_t stream);
constexpr int kDiagFields = 14;

}  // namespace nmhd
