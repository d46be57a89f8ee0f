// Per-cell stage kernels of the B200 ideal-MHD time step, sm_100a: one thread
// per cell on 32 x 4 x 2 CTAs.  Variant 5 (the default): k_cell_flux_staged
// then k_cell_epilogue; variant 4: k_cell_flux then k_cell_epilogue; variant
// 2: k_cell_flux, k_cell_ct, k_cell_prim.
//
//  k_cell_flux  reconstruction + HLLD on the cell's lower x-, y- and z-face
//               (calc_flux_kernel<X,Y,Z>, src/library/mhd_solver.inlrb:562-636);
//               21 flux values per cell go to scratch.
//  k_cell_flux_staged  the same fluxes from a shared-memory copy of the
//               tile's stencil (cell_flux_staged.cuh).
//  k_cell_ct    corner EMFs and the face-B update (:641-714), written into the
//               output state.
//  k_cell_prim  flux divergence (add_flux_kernel :689-693), conserved update
//               (:762-835), primitive recovery (:779-795), the Kepler kick
//               (:837-848), and in the final stage the CFL reduction and clock
//               update (:496-521, 870-901, 981).
//  k_cell_epilogue  k_cell_ct and k_cell_prim fused: one pass per tile with
//               the corner EMFs and new face B in shared memory
//               (cell_epilogue.cuh).
// The per-cell work lives in cell_ops.cuh, shared with the batch kernels.
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "cell_flux_staged.cuh"

// Resident CTAs per SM asked of the compiler (register budget) for the two
// update kernels, both bound by memory latency: measured on the 128x256x64
// box, k_cell_ct is fastest at 4 (64 registers; 5 spills) and k_cell_prim at
// 6 with power-of-two spacings (40 registers, 16 bytes of spill), 4 otherwise
// (no spill).  Staging the CT stencil through a shared-memory tile (34x6x4
// cells, 9 fields) measured no faster than these direct loads.
// k_cell_flux is issue-bound: 4 CTAs/SM (64 registers, 16 bytes of spill) hide
// its fixed-latency waits better than 3 (78 registers): -3 % per launch; 5
// spills 100 bytes and is slower.
#ifndef NMHD_FLUX_MIN_BLOCKS
#define NMHD_FLUX_MIN_BLOCKS 4
#endif
#ifndef NMHD_CT_MIN_BLOCKS
#define NMHD_CT_MIN_BLOCKS 4
#endif
#ifndef NMHD_PRIM_MIN_BLOCKS
#define NMHD_PRIM_MIN_BLOCKS (kPow2 ? 6 : 4)
#endif
// The fused epilogue holds 38.7 KB of shared memory per CTA (5 CTAs/SM).
#ifndef NMHD_EPI_MIN_BLOCKS
#define NMHD_EPI_MIN_BLOCKS 5
#endif
// The staged flux kernel holds 44 KB of shared memory per CTA (4 CTAs/SM).
#ifndef NMHD_SFLUX_MIN_BLOCKS
#define NMHD_SFLUX_MIN_BLOCKS 4
#endif

namespace nmhd {

namespace {

using namespace cell;


// Every kernel covers the z planes [z0, z1) (the whole box, or one chunk of
// the chunked pipeline).
__global__ void __launch_bounds__(kThreads, NMHD_FLUX_MIN_BLOCKS) k_cell_flux(GridParams g, const StepCtl *ctl, const float *w0,
                                                           const float *w1, const float *wp,
                                                           float *__restrict__ flux, int in_sel, int half, int z0,
                                                           int z1) {
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = z0 + blockIdx.z * BZ + threadIdx.z;
  if (x >= g.sx || y >= g.sy || z >= z1) return;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  flux_cell(g, pick(ctl, in_sel, w0, w1, wp), flux, x, y, z, dt);
}

template <bool kPow2>
__global__ void __launch_bounds__(kThreads, NMHD_CT_MIN_BLOCKS) k_cell_ct(GridParams g, const StepCtl *ctl, float *w0,
                                                                          float *w1, float *wp,
                                                                          const float *__restrict__ flux, int in_sel,
                                                                          int out_sel, int half, int z0, int z1) {
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = z0 + blockIdx.z * BZ + threadIdx.z;
  if (x >= g.sx || y >= g.sy || z >= z1) return;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const float *win = pick(ctl, in_sel, w0, w1, wp), *wb = pick(ctl, 0, w0, w1, wp);
  float *wo = const_cast<float *>(pick(ctl, out_sel, w0, w1, wp));
  // CTAs whose cells and their +-1 neighbours all lie inside the box (uniform
  // per CTA) address the neighbours without the periodic wrap
  const int bx0 = blockIdx.x * BX, by0 = blockIdx.y * BY, bz0 = z0 + blockIdx.z * BZ;
  const bool inner = bx0 >= 1 && bx0 + BX < g.sx && by0 >= 1 && by0 + BY < g.sy && bz0 >= 1 && bz0 + BZ < g.sz;
  const int o = (z * g.sy + y) * g.sx + x;
  if (inner)
    ct_core<kPow2>(g, ct_interior(g, win, flux, o), wb, wo, o, dt);
  else
    ct_core<kPow2>(g, ct_global(g, win, flux, x, y, z), wb, wo, o, dt);
}

template <bool kPow2>
__global__ void __launch_bounds__(kThreads, NMHD_PRIM_MIN_BLOCKS) k_cell_prim(GridParams g, StepCtl *ctl, float *w0,
                                                           float *w1, float *wp,
                                                           const float *__restrict__ flux, float *dt_hist,
                                                           int out_sel, int half, int final_stage, int z0,
                                                           int z1, unsigned ntiles) {
  __shared__ float red[kThreads / 32];
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = z0 + blockIdx.z * BZ + threadIdx.z;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  float tcfl = __uint_as_float(0x7f800000u);
  int bad = 0;
  if (x < g.sx && y < g.sy && z < z1)
    tcfl = prim_cell<kPow2>(g, pick(ctl, 0, w0, w1, wp), const_cast<float *>(pick(ctl, out_sel, w0, w1, wp)),
                            flux, x, y, z, dt, final_stage != 0, &bad);
  // ntiles: the CTAs of all this stage's k_cell_prim launches (the last one
  // to finish advances the clock)
  if (final_stage) finish_tile(ctl, ntiles, tcfl, bad, dt_hist, red);
}

// Constrained transport and conserved update of one stage in one pass
// (variant 4); ntiles: the CTAs of this launch (the last one to finish the
// final stage advances the clock).

template <bool kPow2>
__global__ void __launch_bounds__(kThreads, NMHD_EPI_MIN_BLOCKS)
    k_cell_epilogue(const __grid_constant__ epi::EpiMaps maps, GridParams g, StepCtl *ctl, float *w0, float *w1,
                    float *wp, const float *__restrict__ flux, float *dt_hist, int in_sel, int out_sel, int half,
                    int final_stage, unsigned ntiles) {
  __shared__ epi::Smem s;
  if (ctl->done) return;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const float *win = pick(ctl, in_sel, w0, w1, wp), *wb = pick(ctl, 0, w0, w1, wp);
  float *wo = const_cast<float *>(pick(ctl, out_sel, w0, w1, wp));
  int bad = 0, timed_out = 0;
  // tiles in the reverse of the flux kernel's order: CTAs are dispatched in
  // block order, so the first tiles read the fluxes written last, which are
  // still in L2
  const int tx = gridDim.x - 1 - blockIdx.x, ty = gridDim.y - 1 - blockIdx.y, tz = gridDim.z - 1 - blockIdx.z;
  const float tcfl = epi::tile_epilogue<kPow2>(s, g, &maps, pick_index(ctl, in_sel), pick_index(ctl, 0), win, wb, wo,
                                               flux, tx * BX, ty * BY, tz * BZ, dt, final_stage != 0, &bad,
                                               &timed_out);
  if (timed_out && threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0)
    atomicOr(&ctl->status, kStatusTimeout);
  if (final_stage) finish_tile(ctl, ntiles, tcfl, bad, dt_hist, s.red);
}

// Face fluxes of one stage from a shared copy of the stage input (variant
// 5, cell_flux_staged.cuh).
__global__ void __launch_bounds__(kThreads, NMHD_SFLUX_MIN_BLOCKS)
    k_cell_flux_staged(const __grid_constant__ sfx::FluxMaps maps, GridParams g, StepCtl *ctl, const float *w0,
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

dim3 cell_grid(const GridParams &g, int nz) {
  return dim3((g.sx + BX - 1) / BX, (g.sy + BY - 1) / BY, (nz + BZ - 1) / BZ);
}

template <bool kPow2>
void update_range(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux, float *dt_hist,
                  int in_sel, int out_sel, int half, int final_stage, int z0, int z1, unsigned ntiles, bool ct,
                  bool prim, cudaStream_t st) {
  const dim3 grid = cell_grid(g, z1 - z0), blk(BX, BY, BZ);
  if (ct) k_cell_ct<kPow2><<<grid, blk, 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, out_sel, half, z0, z1);
  if (prim)
    k_cell_prim<kPow2><<<grid, blk, 0, st>>>(g, ctl, w0, w1, wp, flux, dt_hist, out_sel, half, final_stage, z0,
                                             z1, ntiles);
}

}  // namespace

void launch_cell_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                      int in_sel, int half, cudaStream_t st) {
  k_cell_flux<<<cell_grid(g, g.sz), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, half, 0, g.sz);
}

void launch_cell_update(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                        float *dt_hist, int in_sel, int out_sel, int half, int final_stage, cudaStream_t st) {
  const dim3 grid = cell_grid(g, g.sz);
  const unsigned ntiles = grid.x * grid.y * grid.z;
  if (g.pow2_spacing)
    update_range<true>(g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half, final_stage, 0, g.sz, ntiles,
                       true, true, st);
  else
    update_range<false>(g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half, final_stage, 0, g.sz, ntiles,
                        true, true, st);
}

// Tensor maps of the fused epilogue's staged boxes for one solver's buffers
// (cuTensorMapEncodeTiled through the runtime's driver entry point): 4-D
// (x, y, z, field) over the 8 state fields or the 21 flux fields, box
// extents the padded shared boxes'.  NULL where the rows are not 16-byte
// multiples (Sx % 4 != 0) or the driver offers no encoder; the kernel then
// stages every tile with cp.async.
EpilogueMaps *make_epilogue_maps(const GridParams &g, float *w0, float *w1, float *wp, float *flux) {
  if (g.sx % 4 != 0) return nullptr;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!encode) return nullptr;
  EpilogueMaps *out = new EpilogueMaps();
  std::memset(out, 0, sizeof(*out));
  const cuuint64_t sx = g.sx, sy = g.sy, sz = g.sz, n = (cuuint64_t)g.n;
  bool ok = true;
  auto make = [&](CUtensorMap *map, float *base, int nfields, int bx, int by, int bz, int bf) {
    const cuuint64_t dims[4] = {sx, sy, sz, (cuuint64_t)nfields};
    const cuuint64_t strides[3] = {sx * 4, sx * sy * 4, n * 4};
    const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, (cuuint32_t)bf};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    ok = ok && encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, es,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  using namespace epi;
  float *w[3] = {w0, w1, wp};
  for (int b = 0; b < 3; ++b) {
    make(&out->m.vel[b], w[b], 8, VelBox::P, VelBox::NJ, VelBox::NK, 3);
    make(&out->m.bx[b], w[b], 8, BXs::P, BXs::NJ, BXs::NK, 1);
    make(&out->m.by[b], w[b], 8, BYs::P, BYs::NJ, BYs::NK, 1);
    make(&out->m.bz[b], w[b], 8, BZs::P, BZs::NJ, BZs::NK, 1);
  }
  make(&out->m.xy, flux, kFluxFields, XYF::P, XYF::NJ, XYF::NK, 1);
  make(&out->m.yx, flux, kFluxFields, YXF::P, YXF::NJ, YXF::NK, 1);
  make(&out->m.xz, flux, kFluxFields, XZF::P, XZF::NJ, XZF::NK, 1);
  make(&out->m.zx, flux, kFluxFields, ZXF::P, ZXF::NJ, ZXF::NK, 1);
  make(&out->m.yz, flux, kFluxFields, YZF::P, YZF::NJ, YZF::NK, 1);
  make(&out->m.zy, flux, kFluxFields, ZYF::P, ZYF::NJ, ZYF::NK, 1);
  for (int b = 0; b < 3; ++b) make(&out->f.w[b], w[b], 8, sfx::P, sfx::NJ, sfx::NK, 8);
  if (!ok) {
    delete out;
    return nullptr;
  }
  out->m.enabled = 1;
  out->f.enabled = 1;
  return out;
}

void free_epilogue_maps(EpilogueMaps *m) { delete m; }

void launch_cell_flux_staged(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                             int in_sel, int half, const EpilogueMaps *maps, cudaStream_t st) {
  static const EpilogueMaps kNone = {};  // enabled = 0: cp.async staging only
  k_cell_flux_staged<<<cell_grid(g, g.sz), dim3(BX, BY, BZ), 0, st>>>(maps ? maps->f : kNone.f, g, ctl, w0, w1,
                                                                      wp, flux, in_sel, half);
}

void launch_cell_update_fused(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                              float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                              const EpilogueMaps *maps, cudaStream_t st) {
  const dim3 grid = cell_grid(g, g.sz), blk(BX, BY, BZ);
  const unsigned ntiles = grid.x * grid.y * grid.z;
  static const EpilogueMaps kNone = {};  // enabled = 0: cp.async staging only
  const epi::EpiMaps &m = maps ? maps->m : kNone.m;
  if (g.pow2_spacing)
    k_cell_epilogue<true><<<grid, blk, 0, st>>>(m, g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half,
                                                final_stage, ntiles);
  else
    k_cell_epilogue<false><<<grid, blk, 0, st>>>(m, g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half,
                                                 final_stage, ntiles);
}

// One RK stage as a z-chunked pipeline (variant 3): chunk c of zc planes is
// reconstructed/solved (F), its face B updated (C) and its cells finished (P)
// so that a chunk's face fluxes are read back while still in L2.  C(c) needs
// F(c-1), F(c), F(c+1) (corner EMFs one plane below and above); P(c) needs
// C(c) and C(c+1) (the new B of the plane above) and F(c), F(c+1).  With the
// periodic wrap the order is F(N-1), F(0), then F(c), C(c-1), P(c-2) for c
// = 1..N-1, then C(N-1), P(N-2), P(N-1).
void launch_cell_stage_chunked(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                               float *dt_hist, int in_sel, int out_sel, int half, int final_stage, int zc,
                               cudaStream_t st) {
  if (zc < 1) zc = g.sz;
  const int nch = (g.sz + zc - 1) / zc;
  auto lo = [&](int c) { return c * zc; };
  auto hi = [&](int c) { return c == nch - 1 ? g.sz : (c + 1) * zc; };
  unsigned ntiles = 0;
  for (int c = 0; c < nch; ++c) {
    const dim3 gr = cell_grid(g, hi(c) - lo(c));
    ntiles += gr.x * gr.y * gr.z;
  }
  const dim3 blk(BX, BY, BZ);
  auto F = [&](int c) {
    k_cell_flux<<<cell_grid(g, hi(c) - lo(c)), blk, 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, half, lo(c), hi(c));
  };
  auto U = [&](int c, bool ct, bool prim) {
    if (g.pow2_spacing)
      update_range<true>(g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half, final_stage, lo(c), hi(c),
                         ntiles, ct, prim, st);
    else
      update_range<false>(g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half, final_stage, lo(c), hi(c),
                          ntiles, ct, prim, st);
  };
  if (nch > 1) F(nch - 1);
  F(0);
  for (int c = 1; c < nch; ++c) {
    if (c < nch - 1) F(c);
    U(c - 1, true, false);
    if (c >= 2) U(c - 2, false, true);
  }
  U(nch - 1, true, false);
  if (nch >= 2) U(nch - 2, false, true);
  U(nch - 1, false, true);
}

}  // namespace nmhd
