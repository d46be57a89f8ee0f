// Batched ensemble: many independent boxes of uneven sizes advanced together.
//
// No counterpart in the reference (one box per process, sizes fixed at compile
// time).  Every box keeps its own configuration, state buffers, control block
// (clock, CFL minimum, status) and therefore its own time step from its own CFL
// reduction.  Each stage kernel of a step is launched over all boxes of a
// launch group (up to 128 boxes, their descriptors in the kernel parameter
// block): a CTA takes a tile of the flattened tile list (or, in the persistent
// schedule, a contiguous range of tiles), finds the tile's box and runs the
// same per-cell code as the single-box path (cell_ops.cuh, margin_ops.cuh,
// cell_flux_staged.cuh, cell_epilogue.cuh), so every box is bitwise the box
// advanced alone.  Each box has its own tile shape; the boxes with the
// single-box kernels' 32 x 4 x 2 tile can run in launches of their own
// (split), through the staged flux and fused update passes.  The launches of
// a step depend on the schedules, not on the number of boxes in a group
// (nmhd_batch_launches_per_step), and batches of steps are one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/nmhd.h"
#include "cell_flux_staged.cuh"
#include "margin_ops.cuh"

namespace nmhd {

struct __align__(8) BoxDesc {
  GridParams g;
  float *w0, *w1, *wp, *flux, *dt_hist;
  StepCtl *ctl;
  // tensor maps of this box's buffers in device memory (boxes with 32 x 4 x 2
  // tiles and Sx % 4 == 0), or NULL: the staged passes then copy by cp.async
  const EpilogueMaps *maps;
  int tile_begin;                 // first tile of this box in the flattened list
  int tiles_x, tiles_y, tiles_z;  // tiles per axis
  int lx, ly, lz;                 // tile of 2^lx x 2^ly x 2^lz cells (256 threads)
  long long fill_begin;           // first Y-margin fill item
  long long mcfl_begin;           // first margin-CFL cell
  long long cell_begin;           // first cell
};

namespace {

using namespace cell;

// Box owning flattened item `i`, where box b owns [begin(b), begin(b+1)).
template <class F>
__device__ __forceinline__ int find_box(int nb, long long i, F begin) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (begin(mid) <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace

// Boxes of one launch group.  The descriptors travel by value in the kernel's
// parameter block (read through the constant bank with a CTA-uniform index), so
// the per-cell code sees its box constants the way the single-box kernels see
// their GridParams argument, without holding them in registers; descriptors
// staged through shared memory cost 16 registers per thread and one resident
// CTA per SM.  Batches of more boxes are split into groups, one launch per
// group and kernel.
constexpr int kGroupBoxes = 128;
struct BatchGroup {
  int nb;                           // boxes in this group
  int total_tiles;                  // tiles of this group
  int fixed_tiles;                  // tiles [0, fixed_tiles): the boxes with 32 x 4 x 2 tiles, placed first
  int tile_begin[kGroupBoxes + 1];  // group-local first tile of each box; [nb] = total_tiles
  BoxDesc box[kGroupBoxes];
};
static_assert(sizeof(BatchGroup) <= 32764, "kernel parameter block limit");

namespace {

// Box of group-local tile t (uniform per CTA).
__device__ __forceinline__ int group_box(const BatchGroup &p, int t) {
  int lo = 0, hi = p.nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.tile_begin[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One tile of one stage kernel: the box's 2^lx x 2^ly x 2^lz cells on the
// CTA's 256 threads (a 1-D block).  KIND 0: face fluxes, 1: constrained
// transport, 2: conserved update + primitive recovery (+ CFL and clock in the
// final stage).
// kFixed: the box has the single-box kernels' 32 x 4 x 2 tile (the shape is
// then a compile-time constant: fewer registers than the general form).
template <int KIND, bool kFixed>
__device__ __forceinline__ void batch_tile(const BoxDesc &d, int t, int in_sel, int out_sel, int half,
                                           int final_stage, float *red) {
  const GridParams &g = d.g;
  StepCtl *ctl = d.ctl;
  const int lx = kFixed ? 5 : d.lx, ly = kFixed ? 2 : d.ly, lz = kFixed ? 1 : d.lz;
  const int lt = t - d.tile_begin;
  const int bx0 = lt % d.tiles_x << lx, by0 = lt / d.tiles_x % d.tiles_y << ly, bz0 = lt / (d.tiles_x * d.tiles_y) << lz;
  const int tid = threadIdx.x;
  const int x = bx0 + (tid & ((1 << lx) - 1)), y = by0 + ((tid >> lx) & ((1 << ly) - 1)), z = bz0 + (tid >> (lx + ly));
  const bool inside = x < g.sx && y < g.sy && z < g.sz;
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  if (KIND == 0) {
    if (inside) flux_cell(g, pick(ctl, in_sel, d.w0, d.w1, d.wp), d.flux, x, y, z, dt);
  } else if (KIND == 1) {
    if (inside) {
      const float *win = pick(ctl, in_sel, d.w0, d.w1, d.wp), *wb = pick(ctl, 0, d.w0, d.w1, d.wp);
      float *wo = const_cast<float *>(pick(ctl, out_sel, d.w0, d.w1, d.wp));
      const int o = (z * g.sy + y) * g.sx + x;
      // tiles whose cells and their +-1 neighbours all lie inside the box
      // address the neighbours without the periodic wrap
      const bool inner = bx0 >= 1 && bx0 + (1 << lx) < g.sx && by0 >= 1 &&
                         by0 + (1 << ly) < g.sy && bz0 >= 1 && bz0 + (1 << lz) < g.sz;
      // always the division form: with power-of-two spacings x / d equals
      // the product form x * (1 / d) bitwise, and one form instead of two
      // keeps the kernel within 64 registers
      if (inner) ct_core<false>(g, ct_interior(g, win, d.flux, o), wb, wo, o, dt);
      else ct_core<false>(g, ct_global_lean(g, win, d.flux, x, y, z), wb, wo, o, dt);
    }
  } else {
    float tcfl = __uint_as_float(0x7f800000u);
    int bad = 0;
    if (inside) {
      const float *wb = pick(ctl, 0, d.w0, d.w1, d.wp);
      float *wo = const_cast<float *>(pick(ctl, out_sel, d.w0, d.w1, d.wp));
      tcfl = g.pow2_spacing ? prim_cell<true>(g, wb, wo, d.flux, x, y, z, dt, final_stage != 0, &bad)
                            : prim_cell<false>(g, wb, wo, d.flux, x, y, z, dt, final_stage != 0, &bad);
    }
    if (final_stage) finish_tile(ctl, (unsigned)(d.tiles_x * d.tiles_y * d.tiles_z), tcfl, bad, d.dt_hist, red);
  }
}

// One stage kernel over tiles [tb, te) of a group, in the schedule that
// nmhd_batch_autotune picks per kernel.  kPersist: a grid of as many CTAs as
// are resident at once, each walking a contiguous range of tiles; otherwise
// one tile per CTA (the default; the hardware scheduler then balances uneven
// tiles across the SMs).  Resident CTAs per SM asked of the compiler:
// NMHD_BATCH_MIN_BLOCKS_<kind>: 4, 3 (4 spills ~100 bytes; the fixed-shape
// form runs 4 with 40 bytes of spill, as the single-box CT kernel), 4.
#ifndef NMHD_BATCH_MIN_BLOCKS_0
#define NMHD_BATCH_MIN_BLOCKS_0 4
#endif
#ifndef NMHD_BATCH_MIN_BLOCKS_1
#define NMHD_BATCH_MIN_BLOCKS_1 3
#endif
#ifndef NMHD_BATCH_MIN_BLOCKS_2
#define NMHD_BATCH_MIN_BLOCKS_2 4
#endif
template <int KIND, bool kPersist, bool kFixed>
__global__ void __launch_bounds__(kThreads, KIND == 0   ? NMHD_BATCH_MIN_BLOCKS_0
                                            : KIND == 1 ? (kFixed ? NMHD_BATCH_MIN_BLOCKS_1 + 1 : NMHD_BATCH_MIN_BLOCKS_1)
                                                        : NMHD_BATCH_MIN_BLOCKS_2)
    k_batch_stage(const __grid_constant__ BatchGroup p, int tb, int te, int in_sel, int out_sel, int half,
                  int final_stage) {
  __shared__ float red[kThreads / 32];
  // this launch's tiles [tb, te): all of the group's, or (split) the
  // fixed-shape boxes' or the others'
  if (!kPersist) {
    const int t = tb + blockIdx.x;
    const BoxDesc &d = p.box[group_box(p, t)];
    if (d.ctl->done) return;
    batch_tile<KIND, kFixed>(d, t, in_sel, out_sel, half, final_stage, red);
    return;
  }
  const int t0 = tb + (int)((long long)(te - tb) * blockIdx.x / gridDim.x);
  const int t1 = tb + (int)((long long)(te - tb) * (blockIdx.x + 1) / gridDim.x);
  int b = group_box(p, t0);
  for (int t = t0; t < t1; ++t) {
    while (t >= p.tile_begin[b + 1]) ++b;
    const BoxDesc &d = p.box[b];
    if (d.ctl->done) continue;
    batch_tile<KIND, kFixed>(d, t, in_sel, out_sel, half, final_stage, red);
  }
}

// Constrained transport and conserved update of the boxes with 32 x 4 x 2
// tiles in one pass per tile: the single-box fused epilogue
// (cell_epilogue.cuh, staging with cp.async), tiles [tb, te) of the group,
// persistent or one tile per CTA.
#ifndef NMHD_BATCH_MIN_BLOCKS_EPI
#define NMHD_BATCH_MIN_BLOCKS_EPI 5
#endif
template <bool kPersist>
__global__ void __launch_bounds__(kThreads, NMHD_BATCH_MIN_BLOCKS_EPI)
    k_batch_epilogue(const __grid_constant__ BatchGroup p, int tb, int te, int in_sel, int out_sel, int half,
                     int final_stage) {
  __shared__ cell::epi::Smem s;
  auto tile = [&](const BoxDesc &d, int t) {
    StepCtl *ctl = d.ctl;
    const int lt = t - d.tile_begin;
    const int x0 = lt % d.tiles_x << 5, y0 = lt / d.tiles_x % d.tiles_y << 2, z0 = lt / (d.tiles_x * d.tiles_y) << 1;
    float dt = step_dt(ctl, nullptr);
    if (half) dt = dt / 2.0f;
    const float *win = pick(ctl, in_sel, d.w0, d.w1, d.wp), *wb = pick(ctl, 0, d.w0, d.w1, d.wp);
    float *wo = const_cast<float *>(pick(ctl, out_sel, d.w0, d.w1, d.wp));
    int bad = 0, timed_out = 0;
    const cell::epi::EpiMaps *maps = d.maps ? &d.maps->m : nullptr;
    const int ib = pick_index(ctl, in_sel), bb = pick_index(ctl, 0);
    const float tcfl =
        d.g.pow2_spacing
            ? cell::epi::tile_epilogue<true>(s, d.g, maps, ib, bb, win, wb, wo, d.flux, x0, y0, z0, dt,
                                            final_stage != 0, &bad, &timed_out)
            : cell::epi::tile_epilogue<false>(s, d.g, maps, ib, bb, win, wb, wo, d.flux, x0, y0, z0, dt,
                                             final_stage != 0, &bad, &timed_out);
    if (timed_out && threadIdx.x == 0) atomicOr(&ctl->status, kStatusTimeout);
    if (final_stage) finish_tile(ctl, (unsigned)(d.tiles_x * d.tiles_y * d.tiles_z), tcfl, bad, d.dt_hist, s.red);
  };
  if (!kPersist) {
    // tiles in the reverse of the flux pass's order (grid = te - tb CTAs,
    // dispatched in block order): the first tiles read the fluxes written
    // last, which are still in L2
    const int t = te - 1 - (int)blockIdx.x;
    const BoxDesc &d = p.box[group_box(p, t)];
    if (d.ctl->done) return;
    tile(d, t);
    return;
  }
  const int t0 = tb + (int)((long long)(te - tb) * blockIdx.x / gridDim.x);
  const int t1 = tb + (int)((long long)(te - tb) * (blockIdx.x + 1) / gridDim.x);
  int b = group_box(p, t0);
  for (int t = t0; t < t1; ++t) {
    while (t >= p.tile_begin[b + 1]) ++b;
    const BoxDesc &d = p.box[b];
    if (d.ctl->done) continue;
    tile(d, t);
    __syncthreads();  // the next tile overwrites the shared tile
  }
}

// Face fluxes of the boxes with 32 x 4 x 2 tiles from a shared copy of each
// tile's stencil: the single-box staged flux kernel (cell_flux_staged.cuh,
// staging with cp.async), tiles [tb, te) of the group, persistent or one
// tile per CTA.
#ifndef NMHD_BATCH_MIN_BLOCKS_SFLUX
#define NMHD_BATCH_MIN_BLOCKS_SFLUX 4
#endif
template <bool kPersist>
__global__ void __launch_bounds__(kThreads, NMHD_BATCH_MIN_BLOCKS_SFLUX)
    k_batch_flux_staged(const __grid_constant__ BatchGroup p, int tb, int te, int in_sel, int half) {
  __shared__ cell::sfx::Smem s;
  const int tid = threadIdx.x;
  const int a = tid % BX, b = tid / BX % BY, c = tid / (BX * BY);
  auto tile = [&](const BoxDesc &d, int t) {
    const GridParams &g = d.g;
    StepCtl *ctl = d.ctl;
    const int lt = t - d.tile_begin;
    const int x0 = lt % d.tiles_x << 5, y0 = lt / d.tiles_x % d.tiles_y << 2, z0 = lt / (d.tiles_x * d.tiles_y) << 1;
    float dt = step_dt(ctl, nullptr);
    if (half) dt = dt / 2.0f;
    if (!cell::sfx::stage(s, g, d.maps ? &d.maps->f : nullptr, pick_index(ctl, in_sel),
                          pick(ctl, in_sel, d.w0, d.w1, d.wp), x0, y0, z0, tid)) {
      if (tid == 0) atomicOr(&ctl->status, kStatusTimeout);
      return;
    }
    const int x = x0 + a, y = y0 + b, z = z0 + c;
    if (x < g.sx && y < g.sy && z < g.sz) cell::sfx::flux_cell_staged(g, s, d.flux, a, b, c, x, y, z, dt);
  };
  if (!kPersist) {
    const int t = tb + blockIdx.x;
    const BoxDesc &d = p.box[group_box(p, t)];
    if (d.ctl->done) return;
    tile(d, t);
    return;
  }
  const int t0 = tb + (int)((long long)(te - tb) * blockIdx.x / gridDim.x);
  const int t1 = tb + (int)((long long)(te - tb) * (blockIdx.x + 1) / gridDim.x);
  int bx = group_box(p, t0);
  for (int t = t0; t < t1; ++t) {
    while (t >= p.tile_begin[bx + 1]) ++bx;
    const BoxDesc &d = p.box[bx];
    if (d.ctl->done) continue;
    tile(d, t);
    __syncthreads();  // the next tile overwrites the shared copy
  }
}

// Shearing-periodic Y-margin fill of every box (margin_ops.cuh).
__global__ void __launch_bounds__(256) k_batch_fill(const BoxDesc *__restrict__ boxes, int nb, long long total) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int b = find_box(nb, i, [&](int k) { return boxes[k].fill_begin; });
    const BoxDesc &d = boxes[b];
    const StepCtl *ctl = d.ctl;
    if (ctl->done) continue;
    float *w = ctl->parity ? d.w1 : d.w0;
    margin::fill_y_item(d.g, ctl->time, w, (int)(i - d.fill_begin));
  }
}

// CFL time of every cell (all = 1) or of the margin cells (all = 0) of every
// box, folded into each box's cfl_cur; lanes of a warp that belong to the same
// box combine before one atomic.
__global__ void __launch_bounds__(256) k_batch_cfl(const BoxDesc *__restrict__ boxes, int nb, long long total,
                                                   int all) {
  for (long long base = (long long)blockIdx.x * blockDim.x; base < total; base += (long long)gridDim.x * blockDim.x) {
    const long long i = base + threadIdx.x;
    int b = -1;
    unsigned bits = 0x7f800000u;
    if (i < total) {
      b = all ? find_box(nb, i, [&](int k) { return boxes[k].cell_begin; })
              : find_box(nb, i, [&](int k) { return boxes[k].mcfl_begin; });
      const BoxDesc &d = boxes[b];
      if (!d.ctl->done) {
        const float *w = d.ctl->parity ? d.w1 : d.w0;
        int x, y, z;
        if (all) {
          const int c = (int)(i - d.cell_begin);
          x = c % d.g.sx;
          y = (c / d.g.sx) % d.g.sy;
          z = c / (d.g.sx * d.g.sy);
        } else {
          margin::margin_cfl_cell(d.g, (int)(i - d.mcfl_begin), &x, &y, &z);
        }
        bits = __float_as_uint(margin::cfl_of_cell(d.g, w, x, y, z));
      }
    }
    const unsigned same = __match_any_sync(0xffffffffu, b);
    const unsigned m = __reduce_min_sync(same, bits);
    const int lane = threadIdx.x & 31;
    if (b >= 0 && lane == __ffs(same) - 1) atomicMin(&boxes[b].ctl->cfl_cur, m);
  }
}

}  // namespace
}  // namespace nmhd

using nmhd::BatchGroup;
using nmhd::BoxDesc;
using nmhd::GridParams;
using nmhd::StepCtl;

struct nmhd_batch {
  int n = 0;
  std::vector<nmhd_config> cfg;
  std::vector<BoxDesc> boxes;
  BoxDesc *d_boxes = nullptr;
  nmhd::EpilogueMaps *d_maps = nullptr;  // per box (used by the boxes whose BoxDesc points here)
  float *pool = nullptr;  // per box: w0, w1, wp (8 fields each), flux (21 fields)
  float *hist = nullptr;
  StepCtl *ctls = nullptr;
  int total_tiles = 0;
  long long total_fill = 0, total_mcfl = 0, total_cells = 0;
  std::vector<nmhd::BatchGroup> groups;  // launch groups of at most kGroupBoxes boxes
  bool persist[3] = {false, false, false};  // schedule of each stage kernel (nmhd_batch_autotune)
  bool split[3] = {true, true, true};       // boxes with 32 x 4 x 2 tiles in a launch of their own
  // with split constrained transport and update: the 32 x 4 x 2 boxes take
  // both in one fused pass (k_batch_epilogue), persistent or one tile per CTA
  bool fuse = false, persist_fused = false;
  // with split face fluxes: the 32 x 4 x 2 boxes' fluxes from a shared copy
  // of each tile's stencil (k_batch_flux_staged), persistent or per tile
  bool sflux = false, persist_sflux = false;
  int ctas[5] = {0, 0, 0, 0, 0};  // resident CTAs of each persistent stage kernel ([3]: fused, [4]: staged flux)
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  bool cfl_ready = false;
  std::map<int, cudaGraphExec_t> graphs;
  // Pinned copies of every box's control block after each of the (at most
  // two) step batches in flight in nmhd_batch_proceed, and their events.
  StepCtl *hctl = nullptr;
  cudaEvent_t batch_done[2] = {nullptr, nullptr};
  std::string err;
};

namespace {

thread_local std::string g_batch_error;

nmhd_status bfail(nmhd_batch *b, nmhd_status st, const std::string &msg) {
  if (b) b->err = msg;
  else g_batch_error = msg;
  return st;
}

#define BATCH_CUDA(b, call)                                                                       \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? NMHD_ERR_OUT_OF_MEMORY : NMHD_ERR_CUDA,   \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                          \
  } while (0)

// Tile shape of a box: the 256 threads of a CTA as 2^lx x 2^ly x 2^lz cells,
// at least 8 wide in x (coalesced rows), chosen to launch the fewest padded
// cells; among equals the widest x, then the shape nearest the single-box
// kernels' 32 x 4 x 2 (stencil neighbours in y and z inside the tile).  Small
// or ragged boxes (e.g. 16 or 48 cells wide) would otherwise idle up to half
// of each warp.
void pick_tile(const GridParams &g, int &lx, int &ly, int &lz) {
  auto padded = [&](int a, int b, int c) {
    return (long long)((g.sx + (1 << a) - 1) >> a << a) * ((g.sy + (1 << b) - 1) >> b << b) *
           ((g.sz + (1 << c) - 1) >> c << c);
  };
  auto key = [&](int a, int b, int c) {
    return std::make_tuple(padded(a, b, c), -a, std::abs(b - 2) + std::abs(c - 1), -b);
  };
  lx = 5, ly = 2, lz = 1;
  for (int a = 5; a >= 3; --a)
    for (int b = 0; a + b <= 8; ++b)
      if (key(a, b, 8 - a - b) < key(lx, ly, lz)) lx = a, ly = b, lz = 8 - a - b;
}

int grid_for(long long work, int cap) {
  long long blocks = (work + 255) / 256;
  return (int)std::max(1LL, std::min<long long>(blocks, cap));
}

template <int KIND>
void launch_stage(const nmhd::BatchGroup &p, bool persist, bool split, int ctas, cudaStream_t st, int in_sel,
                  int out_sel, int half, int fin) {
  const dim3 blk(nmhd::cell::kThreads);
  auto go = [&](auto kernel, int tb, int te) {
    if (te > tb) kernel<<<persist ? std::min(ctas, te - tb) : te - tb, blk, 0, st>>>(p, tb, te, in_sel, out_sel, half, fin);
  };
  if (!split) {  // one launch, every box through the general tile form
    if (persist) go(nmhd::k_batch_stage<KIND, true, false>, 0, p.total_tiles);
    else go(nmhd::k_batch_stage<KIND, false, false>, 0, p.total_tiles);
  } else if (persist) {
    go(nmhd::k_batch_stage<KIND, true, true>, 0, p.fixed_tiles);
    go(nmhd::k_batch_stage<KIND, true, false>, p.fixed_tiles, p.total_tiles);
  } else {
    go(nmhd::k_batch_stage<KIND, false, true>, 0, p.fixed_tiles);
    go(nmhd::k_batch_stage<KIND, false, false>, p.fixed_tiles, p.total_tiles);
  }
}

bool fused(const nmhd_batch *b) { return b->fuse && b->split[1] && b->split[2]; }
bool staged(const nmhd_batch *b) { return b->sflux && b->split[0]; }

// Kernel `kind` of one stage over every group.  Fused: kind 1 covers the
// boxes with general tiles only, kind 2 the fused pass of the 32 x 4 x 2
// boxes and the update of the others.
void launch_kind(nmhd_batch *b, int kind, int in_sel, int out_sel, int half, int fin) {
  const dim3 blk(nmhd::cell::kThreads);
  for (const BatchGroup &p : b->groups) {
    if (kind == 0 && staged(b)) {
      // the other boxes first: the staged pass's fluxes, written last, are
      // the ones the fused pass reads first
      const int tb = p.fixed_tiles, te = p.total_tiles;
      if (te > tb) {
        if (b->persist[0])
          nmhd::k_batch_stage<0, true, false><<<std::min(b->ctas[0], te - tb), blk, 0, b->stream>>>(
              p, tb, te, in_sel, out_sel, half, fin);
        else
          nmhd::k_batch_stage<0, false, false><<<te - tb, blk, 0, b->stream>>>(p, tb, te, in_sel, out_sel, half, fin);
      }
      if (tb > 0) {
        if (b->persist_sflux)
          nmhd::k_batch_flux_staged<true><<<std::min(b->ctas[4], tb), blk, 0, b->stream>>>(p, 0, tb, in_sel, half);
        else
          nmhd::k_batch_flux_staged<false><<<tb, blk, 0, b->stream>>>(p, 0, tb, in_sel, half);
      }
    } else if (kind == 0) {
      launch_stage<0>(p, b->persist[0], b->split[0], b->ctas[0], b->stream, in_sel, out_sel, half, fin);
    } else if (fused(b)) {
      const int tb = p.fixed_tiles, te = p.total_tiles;
      if (kind == 1 && te > tb) {
        if (b->persist[1])
          nmhd::k_batch_stage<1, true, false><<<std::min(b->ctas[1], te - tb), blk, 0, b->stream>>>(
              p, tb, te, in_sel, out_sel, half, fin);
        else
          nmhd::k_batch_stage<1, false, false><<<te - tb, blk, 0, b->stream>>>(p, tb, te, in_sel, out_sel, half, fin);
      }
      if (kind == 2) {
        if (p.fixed_tiles > 0) {
          if (b->persist_fused)
            nmhd::k_batch_epilogue<true><<<std::min(b->ctas[3], p.fixed_tiles), blk, 0, b->stream>>>(
                p, 0, p.fixed_tiles, in_sel, out_sel, half, fin);
          else
            nmhd::k_batch_epilogue<false><<<p.fixed_tiles, blk, 0, b->stream>>>(p, 0, p.fixed_tiles, in_sel,
                                                                                 out_sel, half, fin);
        }
        if (te > tb) {
          if (b->persist[2])
            nmhd::k_batch_stage<2, true, false><<<std::min(b->ctas[2], te - tb), blk, 0, b->stream>>>(
                p, tb, te, in_sel, out_sel, half, fin);
          else
            nmhd::k_batch_stage<2, false, false><<<te - tb, blk, 0, b->stream>>>(p, tb, te, in_sel, out_sel, half, fin);
        }
      }
    } else if (kind == 1) {
      launch_stage<1>(p, b->persist[1], b->split[1], b->ctas[1], b->stream, in_sel, out_sel, half, fin);
    } else {
      launch_stage<2>(p, b->persist[2], b->split[2], b->ctas[2], b->stream, in_sel, out_sel, half, fin);
    }
  }
}

void enqueue_batch_step(nmhd_batch *b) {
  using namespace nmhd;
  cudaStream_t st = b->stream;
  const int cap = 148 * 16;
  if (b->total_fill > 0)
    k_batch_fill<<<grid_for(b->total_fill, cap), 256, 0, st>>>(b->d_boxes, b->n, b->total_fill);
  if (b->total_mcfl > 0)
    k_batch_cfl<<<grid_for(b->total_mcfl, cap), 256, 0, st>>>(b->d_boxes, b->n, b->total_mcfl, 0);
  auto stage = [&](int in_sel, int out_sel, int half, int fin) {
    for (int kind = 0; kind < 3; ++kind) launch_kind(b, kind, in_sel, out_sel, half, fin);
  };
  stage(0, 2, 1, 0);
  stage(2, 1, 0, 1);
}

// Steps per CUDA graph of nmhd_batch_proceed.
constexpr int kBatchSteps = 16;

// The graph of k batched steps (captured on first use).
nmhd_status batch_graph(nmhd_batch *b, int k, cudaGraphExec_t *out) {
  auto it = b->graphs.find(k);
  if (it != b->graphs.end()) {
    *out = it->second;
    return NMHD_OK;
  }
  cudaGraph_t graph;
  cudaGraphExec_t ge;
  BATCH_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < k; ++i) enqueue_batch_step(b);
  BATCH_CUDA(b, cudaStreamEndCapture(b->stream, &graph));
  cudaError_t e = cudaGraphInstantiate(&ge, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return bfail(b, NMHD_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  b->graphs[k] = ge;
  BATCH_CUDA(b, cudaGraphUpload(ge, b->stream));  // the first launch then pays no upload
  *out = ge;
  return NMHD_OK;
}

nmhd_status read_ctls(nmhd_batch *b, std::vector<StepCtl> &h) {
  h.resize(b->n);
  BATCH_CUDA(b, cudaMemcpyAsync(h.data(), b->ctls, sizeof(StepCtl) * b->n, cudaMemcpyDeviceToHost, b->stream));
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  return NMHD_OK;
}

nmhd_status write_ctls(nmhd_batch *b, const std::vector<StepCtl> &h) {
  BATCH_CUDA(b, cudaMemcpyAsync(b->ctls, h.data(), sizeof(StepCtl) * b->n, cudaMemcpyHostToDevice, b->stream));
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  return NMHD_OK;
}

}  // namespace

extern "C" {

nmhd_status nmhd_batch_create(const nmhd_config *cfgs, int n, nmhd_batch **out) {
  if (!out || !cfgs || n < 1) return bfail(nullptr, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  *out = nullptr;
  nmhd_batch *b = new nmhd_batch();
  b->n = n;
  b->cfg.assign(cfgs, cfgs + n);
  // layout: box regions rounded to 64 floats (256 bytes)
  std::vector<size_t> off(n);
  size_t pool_floats = 0;
  for (int i = 0; i < n; ++i) {
    const nmhd_config &c = cfgs[i];
    const long long cells = (long long)c.size_x * c.size_y * c.size_z;
    std::string why;
    const nmhd_status vs = nmhd::validate_config(&c, why);
    if (vs != NMHD_OK) {
      delete b;
      return bfail(nullptr, vs, "box " + std::to_string(i) + ": " + why);
    }
    if (cells * 21 >= (1LL << 31) || c.margin_z != 0 || c.time_order != 2 || c.parallel_size_y > 1 ||
        c.flags != 0) {
      delete b;
      return bfail(nullptr, NMHD_ERR_INVALID_ARGUMENT,
                   "box " + std::to_string(i) + ": invalid configuration (batched boxes are whole boxes with "
                   "time_order 2, no Z margins, flags 0, at most 2^31/21 cells)");
    }
    off[i] = pool_floats;
    pool_floats += (size_t)((cells + 63) / 64 * 64) * (3 * 8 + nmhd::kFluxFields);
  }
  cudaError_t e = cudaGetDevice(&b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&b->pool, sizeof(float) * pool_floats);
  if (e == cudaSuccess) e = cudaMalloc(&b->hist, sizeof(float) * nmhd::kDtHistCap * n);
  if (e == cudaSuccess) e = cudaMalloc(&b->ctls, sizeof(StepCtl) * n);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_boxes, sizeof(BoxDesc) * n);
  if (e == cudaSuccess) e = cudaMallocHost(&b->hctl, 2 * sizeof(StepCtl) * n);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&b->batch_done[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->pool, 0, sizeof(float) * pool_floats, b->stream);
  if (e != cudaSuccess) {
    nmhd_batch_destroy(b);
    return bfail(nullptr, e == cudaErrorMemoryAllocation ? NMHD_ERR_OUT_OF_MEMORY : NMHD_ERR_CUDA,
                 std::string("nmhd_batch_create: ") + cudaGetErrorString(e));
  }
  b->boxes.resize(n);
  std::vector<StepCtl> h(n);
  for (int i = 0; i < n; ++i) {
    BoxDesc &d = b->boxes[i];
    d.g = nmhd::derive_grid(cfgs[i]);
    const size_t cells = (size_t)d.g.n;
    const size_t stride = (cells + 63) / 64 * 64;
    float *base = b->pool + off[i];
    d.w0 = base;
    d.w1 = base + 8 * stride;
    d.wp = base + 16 * stride;
    d.flux = base + 24 * stride;
    d.dt_hist = b->hist + (size_t)nmhd::kDtHistCap * i;
    d.ctl = b->ctls + i;
    pick_tile(d.g, d.lx, d.ly, d.lz);
    d.tiles_x = (d.g.sx + (1 << d.lx) - 1) >> d.lx;
    d.tiles_y = (d.g.sy + (1 << d.ly) - 1) >> d.ly;
    d.tiles_z = (d.g.sz + (1 << d.lz) - 1) >> d.lz;
    d.tile_begin = b->total_tiles;
    d.fill_begin = b->total_fill;
    d.mcfl_begin = b->total_mcfl;
    d.cell_begin = b->total_cells;
    b->total_tiles += d.tiles_x * d.tiles_y * d.tiles_z;
    b->total_fill += (long long)d.g.sx * d.g.my * d.g.sz;
    b->total_mcfl += nmhd::margin::margin_cfl_cells(d.g);
    b->total_cells += (long long)cells;
    std::memset(&h[i], 0, sizeof(StepCtl));
    h[i].cfl_cur = h[i].cfl_next = 0x7f800000u;
    h[i].goal = INFINITY;
    h[i].hist_cap = nmhd::kDtHistCap;
  }
  // tensor maps of the 32 x 4 x 2 boxes' buffers, in device memory: their
  // interior tiles stage by tensor copies as in the single-box kernels
  {
    std::vector<nmhd::EpilogueMaps> hm(n);
    std::memset(hm.data(), 0, sizeof(nmhd::EpilogueMaps) * n);
    std::vector<char> has(n, 0);
    for (int i = 0; i < n; ++i) {
      BoxDesc &d = b->boxes[i];
      d.maps = nullptr;
      if (!(d.lx == 5 && d.ly == 2 && d.lz == 1)) continue;
      nmhd::EpilogueMaps *m = nmhd::make_epilogue_maps(d.g, d.w0, d.w1, d.wp, d.flux);
      if (m) {
        hm[i] = *m;
        has[i] = 1;
        nmhd::free_epilogue_maps(m);
      }
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_maps, sizeof(nmhd::EpilogueMaps) * n);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_maps, hm.data(), sizeof(nmhd::EpilogueMaps) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      for (int i = 0; i < n; ++i)
        if (has[i]) b->boxes[i].maps = b->d_maps + i;
    if (e != cudaSuccess) {
      nmhd_batch_destroy(b);
      return bfail(nullptr, NMHD_ERR_CUDA, std::string("nmhd_batch_create: ") + cudaGetErrorString(e));
    }
  }
  // persistent schedule: as many CTAs as fit on the GPU at once
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  int occ[5] = {1, 1, 1, 1, 1};
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], nmhd::k_batch_stage<0, true, false>, nmhd::cell::kThreads, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], nmhd::k_batch_stage<1, true, false>, nmhd::cell::kThreads, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], nmhd::k_batch_stage<2, true, false>, nmhd::cell::kThreads, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[3], nmhd::k_batch_epilogue<true>, nmhd::cell::kThreads, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[4], nmhd::k_batch_flux_staged<true>, nmhd::cell::kThreads, 0);
  for (int k = 0; k < 5; ++k) b->ctas[k] = sms * std::max(1, occ[k]);
  // launch groups: consecutive boxes, tiles numbered from 0 within a group,
  // the boxes with 32 x 4 x 2 tiles first
  for (int i0 = 0; i0 < n; i0 += nmhd::kGroupBoxes) {
    BatchGroup p;
    std::memset(&p, 0, sizeof p);
    p.nb = std::min(nmhd::kGroupBoxes, n - i0);
    std::vector<int> order;
    for (int pass = 0; pass < 2; ++pass)
      for (int j = 0; j < p.nb; ++j) {
        const BoxDesc &d = b->boxes[i0 + j];
        if ((d.lx == 5 && d.ly == 2 && d.lz == 1) == (pass == 0)) order.push_back(i0 + j);
      }
    for (int j = 0; j < p.nb; ++j) {
      BoxDesc d = b->boxes[order[j]];
      d.tile_begin = p.total_tiles;
      p.box[j] = d;
      p.tile_begin[j] = p.total_tiles;
      p.total_tiles += d.tiles_x * d.tiles_y * d.tiles_z;
      if (d.lx == 5 && d.ly == 2 && d.lz == 1) p.fixed_tiles = p.total_tiles;
    }
    p.tile_begin[p.nb] = p.total_tiles;
    b->groups.push_back(p);
  }
  e = cudaMemcpyAsync(b->d_boxes, b->boxes.data(), sizeof(BoxDesc) * n, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->ctls, h.data(), sizeof(StepCtl) * n, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    nmhd_batch_destroy(b);
    return bfail(nullptr, NMHD_ERR_CUDA, std::string("nmhd_batch_create: ") + cudaGetErrorString(e));
  }
  *out = b;
  return NMHD_OK;
}

void nmhd_batch_destroy(nmhd_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  cudaFree(b->pool);
  cudaFree(b->hist);
  cudaFree(b->ctls);
  cudaFree(b->d_boxes);
  cudaFree(b->d_maps);
  if (b->hctl) cudaFreeHost(b->hctl);
  for (cudaEvent_t ev : b->batch_done)
    if (ev) cudaEventDestroy(ev);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
}

int nmhd_batch_size(const nmhd_batch *b) { return b ? b->n : 0; }

}  // extern "C"

namespace {

// Copies of one box's 8 fields into (to_box) or out of its current buffer,
// whose parity the control block h says.
nmhd_status box_copy(nmhd_batch *b, const StepCtl &h, int box, float *const *fields, int on_device, bool to_box) {
  const BoxDesc &d = b->boxes[box];
  float *cur = h.parity ? d.w1 : d.w0;
  const size_t bytes = sizeof(float) * (size_t)d.g.n;
  for (int v = 0; v < 8; ++v) {
    if (!fields[v]) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "field pointer is NULL");
    float *dev = cur + (size_t)v * d.g.n;
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice
                                          : (to_box ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost);
    BATCH_CUDA(b, cudaMemcpyAsync(to_box ? dev : fields[v], to_box ? fields[v] : dev, bytes, kind, b->stream));
  }
  return NMHD_OK;
}

// States of boxes [b0, b1) in (fields box-major, 8 per box): one round trip
// to the control blocks for all of them.
nmhd_status set_states(nmhd_batch *b, int b0, int b1, const float *const *fields, int on_device) {
  std::vector<StepCtl> h;
  nmhd_status st = read_ctls(b, h);
  if (st != NMHD_OK) return st;
  for (int box = b0; box < b1; ++box) {
    st = box_copy(b, h[box], box, const_cast<float *const *>(fields + 8 * (box - b0)), on_device, true);
    if (st != NMHD_OK) return st;
    h[box].status = 0;
    h[box].done = 0;
    h[box].cfl_cur = h[box].cfl_next = 0x7f800000u;
  }
  b->cfl_ready = false;
  return write_ctls(b, h);
}

nmhd_status get_states(nmhd_batch *b, int b0, int b1, float *const *fields, int on_device) {
  std::vector<StepCtl> h;
  nmhd_status st = read_ctls(b, h);
  if (st != NMHD_OK) return st;
  for (int box = b0; box < b1; ++box) {
    st = box_copy(b, h[box], box, fields + 8 * (box - b0), on_device, false);
    if (st != NMHD_OK) return st;
  }
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  return NMHD_OK;
}

}  // namespace

extern "C" {

nmhd_status nmhd_batch_set_state(nmhd_batch *b, int box, const float *const fields[8], int on_device) {
  if (!b || !fields || box < 0 || box >= b->n) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  return set_states(b, box, box + 1, fields, on_device);
}

nmhd_status nmhd_batch_get_state(nmhd_batch *b, int box, float *const fields[8], int on_device) {
  if (!b || !fields || box < 0 || box >= b->n) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  return get_states(b, box, box + 1, fields, on_device);
}

nmhd_status nmhd_batch_set_states(nmhd_batch *b, const float *const *fields, int on_device) {
  if (!b || !fields) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  return set_states(b, 0, b->n, fields, on_device);
}

nmhd_status nmhd_batch_get_states(nmhd_batch *b, float *const *fields, int on_device) {
  if (!b || !fields) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  return get_states(b, 0, b->n, fields, on_device);
}

nmhd_status nmhd_batch_clock(nmhd_batch *b, int box, double *time, int64_t *generation) {
  if (!b || box < 0 || box >= b->n) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  std::vector<StepCtl> h;
  nmhd_status st = read_ctls(b, h);
  if (st != NMHD_OK) return st;
  if (time) *time = h[box].time;
  if (generation) *generation = h[box].generation;
  return NMHD_OK;
}

nmhd_status nmhd_batch_proceed(nmhd_batch *b, double goal_time, int64_t max_steps, int64_t *steps_done) {
  if (steps_done) *steps_done = 0;
  if (!b) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "NULL batch");
  std::vector<StepCtl> h;
  nmhd_status st = read_ctls(b, h);
  if (st != NMHD_OK) return st;
  for (int i = 0; i < b->n; ++i)
    if (h[i].status) return bfail(b, NMHD_ERR_NUMERICAL, "box " + std::to_string(i) + " holds an invalid state");
  long long gen0 = 0;
  for (int i = 0; i < b->n; ++i) {
    gen0 = std::max(gen0, h[i].generation);
    h[i].goal = (float)goal_time;
    h[i].done = 0;
    if (!b->cfl_ready) {
      h[i].cfl_cur = h[i].cfl_next = 0x7f800000u;
      h[i].blocks_done = 0;
    }
  }
  st = write_ctls(b, h);
  if (st != NMHD_OK) return st;
  if (!b->cfl_ready) {
    const int cap = 148 * 16;
    if (b->total_fill > 0)
      nmhd::k_batch_fill<<<grid_for(b->total_fill, cap), 256, 0, b->stream>>>(b->d_boxes, b->n, b->total_fill);
    nmhd::k_batch_cfl<<<grid_for(b->total_cells, cap), 256, 0, b->stream>>>(b->d_boxes, b->n, b->total_cells, 1);
    BATCH_CUDA(b, cudaGetLastError());
    b->cfl_ready = true;
  }
  // As nmhd_proceed: batches of kBatchSteps steps, one graph each, the next
  // launched before the previous one's control blocks are read (a batch
  // after every box's goal step returns at once on the device).
  long long left = max_steps > 0 ? max_steps : -1;
  int queue[2], queued = 0, head = 0, next_slot = 0;
  const size_t nctl = (size_t)b->n;
  nmhd_status result = NMHD_OK;
  for (;;) {
    while (queued < 2 && left != 0) {
      int k = kBatchSteps;
      if (left >= 0 && left < k) k = (int)left;
      cudaGraphExec_t ge;
      st = batch_graph(b, k, &ge);
      if (st != NMHD_OK) return st;
      const int slot = next_slot;
      next_slot ^= 1;
      BATCH_CUDA(b, cudaGraphLaunch(ge, b->stream));
      BATCH_CUDA(b, cudaMemcpyAsync(b->hctl + slot * nctl, b->ctls, sizeof(StepCtl) * nctl,
                                    cudaMemcpyDeviceToHost, b->stream));
      BATCH_CUDA(b, cudaEventRecord(b->batch_done[slot], b->stream));
      queue[(head + queued) % 2] = slot;
      ++queued;
      if (left > 0) left -= k;
    }
    if (queued == 0) { result = NMHD_STEP_LIMIT; break; }
    const int slot = queue[head];
    head = (head + 1) % 2;
    --queued;
    BATCH_CUDA(b, cudaEventSynchronize(b->batch_done[slot]));
    h.assign(b->hctl + slot * nctl, b->hctl + (slot + 1) * nctl);
    int bad = -1, done = 0;
    for (int i = 0; i < b->n; ++i) {
      if (h[i].status && bad < 0) bad = i;
      done += h[i].done;
    }
    if (bad >= 0) {
      result = bfail(b, NMHD_ERR_NUMERICAL, "box " + std::to_string(bad) + ": non-finite state, density <= 0, "
                                            "pressure <= 0 or bad dt");
      break;
    }
    if (done == b->n) { result = NMHD_GOAL_REACHED; break; }
  }
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  if (steps_done) {
    long long gen1 = 0;
    for (int i = 0; i < b->n; ++i) gen1 = std::max(gen1, h[i].generation);
    *steps_done = gen1 - gen0;
  }
  return result;
}

nmhd_status nmhd_batch_prepare(nmhd_batch *b, int64_t max_steps) {
  if (!b) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "NULL batch");
  cudaGraphExec_t ge;
  const int first = max_steps > 0 && max_steps < kBatchSteps ? (int)max_steps : kBatchSteps;
  nmhd_status st = batch_graph(b, first, &ge);
  if (st == NMHD_OK && max_steps > kBatchSteps && max_steps % kBatchSteps)
    st = batch_graph(b, (int)(max_steps % kBatchSteps), &ge);
  return st;
}

int nmhd_batch_launches_per_step(const nmhd_batch *b) {
  if (!b) return NMHD_ERR_INVALID_ARGUMENT;
  int n = (b->total_fill > 0) + (b->total_mcfl > 0);
  for (const BatchGroup &p : b->groups) {
    const int fixed = p.fixed_tiles > 0, general = p.total_tiles > p.fixed_tiles;
    n += 2 * (b->split[0] ? fixed + general : 1);
    if (fused(b))  // per stage: CT of the general boxes, the fused pass, the general update
      n += 2 * (general + fixed + general);
    else
      for (int kind = 1; kind < 3; ++kind) n += 2 * (b->split[kind] ? fixed + general : 1);
  }
  return n;
}

nmhd_status nmhd_batch_tile_rule(const nmhd_config *box, int *tile_x, int *tile_y, int *tile_z) {
  if (!box || box->size_x < 1 || box->size_y < 1 || box->size_z < 1) return NMHD_ERR_INVALID_ARGUMENT;
  int lx, ly, lz;
  pick_tile(nmhd::derive_grid(*box), lx, ly, lz);
  if (tile_x) *tile_x = 1 << lx;
  if (tile_y) *tile_y = 1 << ly;
  if (tile_z) *tile_z = 1 << lz;
  return NMHD_OK;
}

nmhd_status nmhd_batch_set_stream(nmhd_batch *b, void *cuda_stream) {
  if (!b) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "NULL batch");
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  if (b->own_stream) cudaStreamDestroy(b->stream);
  b->stream = nullptr;
  b->own_stream = cuda_stream == nullptr;
  if (b->own_stream) BATCH_CUDA(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  else b->stream = (cudaStream_t)cuda_stream;
  return NMHD_OK;
}

nmhd_status nmhd_batch_tile_shape(const nmhd_batch *b, int box, int *tile_x, int *tile_y, int *tile_z) {
  if (!b || box < 0 || box >= b->n) return NMHD_ERR_INVALID_ARGUMENT;
  const BoxDesc &d = b->boxes[box];
  if (tile_x) *tile_x = 1 << d.lx;
  if (tile_y) *tile_y = 1 << d.ly;
  if (tile_z) *tile_z = 1 << d.lz;
  return NMHD_OK;
}

nmhd_status nmhd_batch_set_schedule(nmhd_batch *b, int kernel, int persistent, int split) {
  if (!b || kernel < 0 || kernel > 4 || (persistent != 0 && persistent != 1) || (split != 0 && split != 1))
    return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "kernel must be 0..4, persistent and split 0 or 1");
  BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
  if (kernel == 3) {  // the fused pass: on (split = 1) or off, and its schedule
    b->fuse = split != 0;
    b->persist_fused = persistent != 0;
  } else if (kernel == 4) {  // the staged flux pass: on (split = 1) or off, and its schedule
    b->sflux = split != 0;
    b->persist_sflux = persistent != 0;
  } else {
    b->persist[kernel] = persistent != 0;
    b->split[kernel] = split != 0;
  }
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  return NMHD_OK;
}

int nmhd_batch_autotune(nmhd_batch *b, int reps, double *trials_out, int max_trials) {
  if (!b || reps <= 0) return bfail(b, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  std::vector<StepCtl> h0;
  nmhd_status st = read_ctls(b, h0);
  if (st != NMHD_OK) return st;
  for (int i = 0; i < b->n; ++i)
    if (h0[i].status) return bfail(b, NMHD_ERR_NUMERICAL, "box " + std::to_string(i) + " holds an invalid state");
  // every box live, with the CFL time step of its current state
  std::vector<StepCtl> h = h0;
  for (StepCtl &c : h) {
    c.goal = INFINITY;
    c.done = 0;
    if (!b->cfl_ready) {
      c.cfl_cur = c.cfl_next = 0x7f800000u;
      c.blocks_done = 0;
    }
  }
  st = write_ctls(b, h);
  if (st != NMHD_OK) return st;
  const int cap = 148 * 16;
  if (!b->cfl_ready) {
    if (b->total_fill > 0)
      nmhd::k_batch_fill<<<grid_for(b->total_fill, cap), 256, 0, b->stream>>>(b->d_boxes, b->n, b->total_fill);
    nmhd::k_batch_cfl<<<grid_for(b->total_cells, cap), 256, 0, b->stream>>>(b->d_boxes, b->n, b->total_cells, 1);
  }
  // The first stage's kernels (state -> fluxes -> predictor) leave the state
  // and the clocks alone, so each can be launched again and again on it.
  const bool saved[3] = {b->persist[0], b->persist[1], b->persist[2]};
  const bool saved_split[3] = {b->split[0], b->split[1], b->split[2]};
  const bool saved_fuse = b->fuse, saved_pf = b->persist_fused;
  const bool saved_sflux = b->sflux, saved_ps = b->persist_sflux;
  b->fuse = false;  // each kernel alone first; the fused passes are compared last
  b->sflux = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  for (int kind = 0; kind < 3 && e == cudaSuccess; ++kind) launch_kind(b, kind, 0, 2, 1, 0);
  int written = 0;
  for (int kind = 0; kind < 3 && e == cudaSuccess; ++kind) {
    double best = 1e30;
    bool choice = saved[kind], choice_split = saved_split[kind];
    for (int trial = 0; trial < 4 && e == cudaSuccess; ++trial) {
      const int persist = trial & 1, split = trial >> 1;
      b->persist[kind] = persist != 0;
      b->split[kind] = split != 0;
      launch_kind(b, kind, 0, 2, 1, 0);  // warm-up
      e = cudaEventRecord(e0, b->stream);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) launch_kind(b, kind, 0, 2, 1, 0);
      if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) break;
      const double per = ms / reps;
      if (trials_out && written < max_trials) {
        trials_out[4 * written + 0] = kind;
        trials_out[4 * written + 1] = persist;
        trials_out[4 * written + 2] = split;
        trials_out[4 * written + 3] = per;
        ++written;
      }
      if (per < best) {
        best = per;
        choice = persist != 0;
        choice_split = split != 0;
      }
    }
    b->persist[kind] = choice;
    b->split[kind] = choice_split;
  }
  // The face fluxes with the chosen schedule against the staged flux pass for
  // the 32 x 4 x 2 boxes (fluxes split), one tile per CTA or persistent:
  // rows (4, persistent, staged, ms per launch).
  {
    const bool keep_split = b->split[0];
    double best = 1e30;
    bool best_on = false, best_p = false, any_fixed = false;
    for (const BatchGroup &p : b->groups) any_fixed = any_fixed || p.fixed_tiles > 0;
    for (int trial = 0; trial < 3 && e == cudaSuccess; ++trial) {
      const int on = trial > 0, ps = trial == 2;
      if (on && !any_fixed) break;
      b->sflux = on != 0;
      b->persist_sflux = ps != 0;
      if (on) b->split[0] = true;
      launch_kind(b, 0, 0, 2, 1, 0);  // warm-up
      e = cudaEventRecord(e0, b->stream);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) launch_kind(b, 0, 0, 2, 1, 0);
      if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) break;
      const double per = ms / reps;
      if (trials_out && written < max_trials) {
        trials_out[4 * written + 0] = 4;
        trials_out[4 * written + 1] = ps;
        trials_out[4 * written + 2] = on;
        trials_out[4 * written + 3] = per;
        ++written;
      }
      if (per < best) {
        best = per;
        best_on = on != 0;
        best_p = ps != 0;
      }
      if (on) b->split[0] = keep_split;
    }
    b->sflux = best_on;
    b->persist_sflux = best_p;
    if (best_on) b->split[0] = true;
  }
  // The stage's update (constrained transport, then conserved update) with
  // the chosen schedules, against the fused pass for the 32 x 4 x 2 boxes
  // (both kernels split), one tile per CTA or persistent: rows of kernel 3,
  // (3, persistent, fused, ms per update).
  {
    const bool keep_split[2] = {b->split[1], b->split[2]};
    double best = 1e30;
    bool best_fuse = false, best_pf = false, any_fixed = false;
    for (const BatchGroup &p : b->groups) any_fixed = any_fixed || p.fixed_tiles > 0;
    for (int trial = 0; trial < 3 && e == cudaSuccess; ++trial) {
      const int f = trial > 0, pf = trial == 2;
      if (f && !any_fixed) break;
      b->fuse = f != 0;
      b->persist_fused = pf != 0;
      if (f) b->split[1] = b->split[2] = true;
      launch_kind(b, 1, 0, 2, 1, 0);  // warm-up
      launch_kind(b, 2, 0, 2, 1, 0);
      e = cudaEventRecord(e0, b->stream);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        launch_kind(b, 1, 0, 2, 1, 0);
        launch_kind(b, 2, 0, 2, 1, 0);
      }
      if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) break;
      const double per = ms / reps;
      if (trials_out && written < max_trials) {
        trials_out[4 * written + 0] = 3;
        trials_out[4 * written + 1] = pf;
        trials_out[4 * written + 2] = f;
        trials_out[4 * written + 3] = per;
        ++written;
      }
      if (per < best) {
        best = per;
        best_fuse = f != 0;
        best_pf = pf != 0;
      }
      if (f) b->split[1] = keep_split[0], b->split[2] = keep_split[1];
    }
    b->fuse = best_fuse;
    b->persist_fused = best_pf;
    if (best_fuse) b->split[1] = b->split[2] = true;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    for (int k = 0; k < 3; ++k) b->persist[k] = saved[k], b->split[k] = saved_split[k];
    b->fuse = saved_fuse;
    b->persist_fused = saved_pf;
    b->sflux = saved_sflux;
    b->persist_sflux = saved_ps;
    return bfail(b, NMHD_ERR_CUDA, std::string("nmhd_batch_autotune: ") + cudaGetErrorString(e));
  }
  // the graphs hold the previous schedules
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  st = write_ctls(b, h0);  // clocks, goals and CFL minima as they were
  if (st != NMHD_OK) return st;
  return written;
}

const char *nmhd_batch_last_error(const nmhd_batch *b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

}  // extern "C"
