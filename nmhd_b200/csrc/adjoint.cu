// Differentiation of the B200 time step (sm_100a): FP32 and FP64 adjoint runs
// with checkpointed recomputation, and the FP64 tangent-linear run.
//
// FP32 runs step with the production kernels (cell_stage.cu) on explicit
// buffers, so the forward trajectory, its CFL time steps and its loss are
// bitwise those of nmhd_proceed; the dt is then frozen through StepCtl::dt_seq
// for the recomputation.  FP64 and tangent-linear runs step with the generic
// kernels of ad_driver.cuh over double and Dual<double>.  The adjoint kernels
// are the transposes in ad_cell.cuh / ad_hlld.cuh, one launch per pass.
//
// Memory: checkpoints (8 fields) every K steps, plus the tape (24 fields per
// step: filled input, predictor, raw output) of the last segments, one shared
// 21-field flux scratch, plus 3 adjoint states and 42 scratch fields.  The forward run
// keeps as many trailing segments on the tape as the tape budget allows (at
// least one; by default as many as fit in half of the free device memory),
// and the reverse sweep recomputes only the earlier segments, from their
// checkpoints.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/nmhd.h"
#include "ad_driver.cuh"
#include "solver_impl.h"
#include "step.cuh"

using nmhd::GridParams;
using nmhd::StepCtl;
using namespace nmhd::ad;

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

// Resident CTAs per SM asked of the compiler: the FP32 HLLD adjoint is
// latency-bound at one 256-thread CTA per SM, so it is held to 128 registers
// (2 CTAs).
template <class F>
struct MinBlocks {
  static constexpr int value = 1;
};
template <int AX>
struct MinBlocks<OpAFlux<float, AX>> {
  static constexpr int value = 2;
};
// The gather passes (reconstruction transposes, primitive and face-B
// adjoints) are bound by memory latency: 8 CTAs/SM (32 registers, no spill)
// took the adjoint kernels from 72.6 to 68.6 ms on 64^3 x 200 steps; 6 gained
// nothing.
#ifndef NMHD_AD_GATHER_MIN_BLOCKS
#define NMHD_AD_GATHER_MIN_BLOCKS 8
#endif
template <int AX>
struct MinBlocks<OpARecon<float, AX>> {
  static constexpr int value = NMHD_AD_GATHER_MIN_BLOCKS;
};
template <>
struct MinBlocks<OpAPrim<float>> {
  static constexpr int value = NMHD_AD_GATHER_MIN_BLOCKS;
};
template <>
struct MinBlocks<OpABface<float>> {
  static constexpr int value = NMHD_AD_GATHER_MIN_BLOCKS;
};

// Programmatic dependent launch: the executor launches each pass so that it
// may be scheduled while the previous pass's last blocks still run; every
// pass lets its own successor be scheduled at once, then waits until the
// previous grid has completed and its memory is visible, before its first
// global access.  (Both are no-ops for a launch without the attribute.)
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <class F, int kMinBlocks>
__global__ void __launch_bounds__(BX *BY *BZ, kMinBlocks) k_ad_cells(F f, int sx, int sy, int sz) {
  pdl_enter();
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = blockIdx.z * BZ + threadIdx.z;
  if (x < sx && y < sy && z < sz) f(x, y, z);
}

template <class F>
__global__ void __launch_bounds__(256) k_ad_items(F f, int n) {
  pdl_enter();
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i < n) f(i);
}

// Deterministic reduction of a per-cell value: a fixed tree per block into
// partial[], then one block folds partial[] in a fixed order into *acc.
template <class D, class F>
__global__ void __launch_bounds__(256) k_ad_reduce(F f, int sx, int sy, int sz, D *partial) {
  __shared__ double raw[256 * sizeof(D) / sizeof(double)];
  D *sh = reinterpret_cast<D *>(raw);
  pdl_enter();
  const int tid = threadIdx.x;
  const long long i = (long long)blockIdx.x * 256 + tid;
  const long long n = (long long)sx * sy * sz;
  D v = to<D>(0.0);
  if (i < n) {
    const int x = (int)(i % sx), y = (int)((i / sx) % sy), z = (int)(i / ((long long)sx * sy));
    v = f(x, y, z);
  }
  sh[tid] = v;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (tid < s) sh[tid] = sh[tid] + sh[tid + s];
    __syncthreads();
  }
  if (tid == 0) partial[blockIdx.x] = sh[0];
}

template <class D>
__global__ void __launch_bounds__(256) k_ad_reduce_final(const D *partial, int nb, D *acc, double scale) {
  __shared__ double raw[256 * sizeof(D) / sizeof(double)];
  D *sh = reinterpret_cast<D *>(raw);
  pdl_enter();
  const int tid = threadIdx.x;
  D v = to<D>(0.0);
  for (int i = tid; i < nb; i += 256) v = v + partial[i];
  sh[tid] = v;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (tid < s) sh[tid] = sh[tid] + sh[tid + s];
    __syncthreads();
  }
  if (tid == 0) acc[0] = acc[0] + sh[0] * to<D>(scale);
}

template <class T>
struct OpWiden {  // float state (+ shift * dir) -> T, with dir as the tangent
  const float *src;
  const double *dir;
  double shift;
  T *dst;
  NMHD_HD void operator()(int i) const;
};
template <>
NMHD_HD void OpWiden<double>::operator()(int i) const { dst[i] = (double)src[i]; }
template <>
NMHD_HD void OpWiden<Dual<double>>::operator()(int i) const {
  dst[i] = dir ? Dual<double>((double)src[i] + shift * dir[i], dir[i]) : Dual<double>((double)src[i], 0.0);
}

// Launch with programmatic stream serialization (see pdl_enter).
template <class... KArgs, class... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

struct GpuExec {
  cudaStream_t st;
  template <class R, class F>
  void cells(const GGrid<R> &g, const F &f) {
    const dim3 grid((g.sx + BX - 1) / BX, (g.sy + BY - 1) / BY, (g.sz + BZ - 1) / BZ);
    launch_pdl(k_ad_cells<F, MinBlocks<F>::value>, grid, dim3(BX, BY, BZ), st, f, g.sx, g.sy, g.sz);
  }
  template <class F>
  void items(int n, const F &f) {
    if (n > 0) launch_pdl(k_ad_items<F>, dim3((n + 255) / 256), dim3(256), st, f, n);
  }
  template <class T>
  void zero(T *p, size_t n) {
    cudaMemsetAsync(p, 0, n * sizeof(T), st);
  }
  template <class D, class R, class F>
  void reduce(const GGrid<R> &g, const F &f, D *partial, D *acc, double scale) {
    const long long n = (long long)g.sx * g.sy * g.sz;
    const int nb = (int)((n + 255) / 256);
    launch_pdl(k_ad_reduce<D, F>, dim3(nb), dim3(256), st, f, g.sx, g.sy, g.sz, partial);
    launch_pdl(k_ad_reduce_final<D>, dim3(1), dim3(256), st, (const D *)partial, nb, acc, scale);
  }
};

// ---------------------------------------------------------------------------
struct Workspace {
  void *mem = nullptr;
  size_t bytes = 0;
  long long tape_budget = -1;  // bytes for the tapes of segments beyond the last; -1: automatic
  int parity = 0;              // StepCtl::parity as the production steps leave it (host copy)
  int kept_segments = 0;       // of the last run
  StepCtl *ctl = nullptr;
  float *dt_dev = nullptr, *hist_dummy = nullptr;
  double ms[4] = {0, 0, 0, 0};
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // Segment recomputation runs on a stream of its own, beside the reverse
  // sweep: control blocks are staged in pinned memory (one per segment, so
  // none is overwritten before its copy runs) and two tape slots alternate,
  // ordered by "slot recomputed" / "slot swept" events.
  // The reverse sweep itself runs on stream_hi, at the device's highest
  // stream priority, the recomputation on stream2 at the lowest: the sweep's
  // thread blocks are scheduled first and the recomputation fills the SMs
  // they leave free.
  cudaStream_t stream2 = nullptr, stream_hi = nullptr;
  StepCtl *hstage = nullptr;  // pinned, NMHD_ADJOINT_MAX_STEPS entries
  cudaEvent_t slot_ready[2] = {nullptr, nullptr}, slot_free[2] = {nullptr, nullptr}, fwd_done = nullptr,
              sweep_done = nullptr;
  // Tensor maps of the production kernels for each (w0, w1, predictor, flux)
  // buffer set a taped step runs on, made on first use: the sets are fixed
  // while the arena stays, so repeated runs reuse them.
  std::map<std::array<const void *, 4>, nmhd::EpilogueMaps *> maps;
  void clear_maps() {
    for (auto &kv : maps) nmhd::free_epilogue_maps(kv.second);
    maps.clear();
  }
};

Workspace &workspace(nmhd_solver *s) {
  if (!s->adjoint) s->adjoint = new Workspace();
  return *static_cast<Workspace *>(s->adjoint);
}

nmhd_status set_err(nmhd_solver *s, nmhd_status st, const std::string &m) {
  s->err = m;
  return st;
}

#define AD_CUDA(call)                                                                                \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return set_err(s, e_ == cudaErrorMemoryAllocation ? NMHD_ERR_OUT_OF_MEMORY : NMHD_ERR_CUDA,    \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                            \
  } while (0)

// One arena per run: the run's buffers are carved from it in order.  A dry
// run with base 0 measures the bytes the same carve sequence needs.
struct Arena {
  uintptr_t base;
  size_t off;
  template <class T>
  T *take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T *p = reinterpret_cast<T *>(base + off);
    off += count * sizeof(T);
    return p;
  }
};

nmhd_status reserve(nmhd_solver *s, Workspace &w, size_t bytes) {
  if (!w.ctl) {
    AD_CUDA(cudaMalloc(&w.ctl, sizeof(StepCtl)));
    AD_CUDA(cudaMalloc(&w.dt_dev, sizeof(float) * nmhd::kDtHistCap));
    AD_CUDA(cudaMalloc(&w.hist_dummy, sizeof(float) * nmhd::kDtHistCap));
    for (auto &e : w.ev) AD_CUDA(cudaEventCreate(&e));
    int prio_low = 0, prio_high = 0;
    AD_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    AD_CUDA(cudaStreamCreateWithPriority(&w.stream2, cudaStreamNonBlocking, prio_low));
    AD_CUDA(cudaStreamCreateWithPriority(&w.stream_hi, cudaStreamNonBlocking, prio_high));
    AD_CUDA(cudaMallocHost(&w.hstage, sizeof(StepCtl) * NMHD_ADJOINT_MAX_STEPS));
    for (int i = 0; i < 2; ++i) {
      AD_CUDA(cudaEventCreateWithFlags(&w.slot_ready[i], cudaEventDisableTiming));
      AD_CUDA(cudaEventCreateWithFlags(&w.slot_free[i], cudaEventDisableTiming));
    }
    AD_CUDA(cudaEventCreateWithFlags(&w.fwd_done, cudaEventDisableTiming));
    AD_CUDA(cudaEventCreateWithFlags(&w.sweep_done, cudaEventDisableTiming));
  }
  if (w.bytes >= bytes) return NMHD_OK;
  if (w.mem) {
    AD_CUDA(cudaStreamSynchronize(s->stream));
    cudaFree(w.mem);
    w.mem = nullptr;
    w.bytes = 0;
    w.clear_maps();  // they name the old arena's buffers
  }
  AD_CUDA(cudaMalloc(&w.mem, bytes));
  w.bytes = bytes;
  return NMHD_OK;
}

nmhd_status validate(nmhd_solver *s, int nsteps, int ckpt, const nmhd_loss_spec *l) {
  if (!s) return NMHD_ERR_INVALID_ARGUMENT;
  if (!l) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "loss spec is NULL");
  if (nsteps < 1 || nsteps > NMHD_ADJOINT_MAX_STEPS)
    return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "nsteps must be in [1, NMHD_ADJOINT_MAX_STEPS]");
  if (ckpt < 1) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "ckpt_every must be >= 1");
  if (l->kind != NMHD_LOSS_MAXWELL_STRESS) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "unknown loss kind");
  if (l->first_step < 0 || l->first_step > l->last_step || l->last_step > nsteps)
    return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "loss window must satisfy 0 <= first <= last <= nsteps");
  if (s->cfg.size_y - 2 * s->cfg.margin_y < 1 || s->cfg.size_z - 2 * s->cfg.margin_z < 1)
    return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "no interior cells");
  if (s->cfg.parallel_size_y > 1)
    return set_err(s, NMHD_ERR_NOT_SUPPORTED, "the differentiated step covers a whole box, not a radial slab");
  if (s->cfg.flags)
    return set_err(s, NMHD_ERR_NOT_SUPPORTED, "the differentiated step is the reference's scheme (flags 0)");
  return NMHD_OK;
}

// The solver's current state (device) and clock.
nmhd_status solver_state(nmhd_solver *s, const float **cur, double *time) {
  StepCtl h;
  AD_CUDA(cudaMemcpyAsync(&h, s->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s->stream));
  AD_CUDA(cudaStreamSynchronize(s->stream));
  if (h.status) return set_err(s, NMHD_ERR_NUMERICAL, "state is not valid (set a new state)");
  *cur = h.parity ? s->w1 : s->w0;
  *time = h.time;
  return NMHD_OK;
}

nmhd_status write_ctl(nmhd_solver *s, Workspace &w, double time, long long gen, bool frozen) {
  StepCtl h;
  std::memset(&h, 0, sizeof(h));
  h.time = time;
  h.generation = gen;
  h.cfl_cur = h.cfl_next = 0x7f800000u;
  h.goal = INFINITY;
  h.hist_cap = nmhd::kDtHistCap;
  h.dt_seq = frozen ? w.dt_dev : nullptr;
  h.dt_seq_base = 0;
  w.parity = 0;
  AD_CUDA(cudaMemcpyAsync(w.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s->stream));
  AD_CUDA(cudaStreamSynchronize(s->stream));
  return NMHD_OK;
}

// The same control block for the recomputation of segment `slot` (an index
// into the pinned staging array), copied on `stream` without a host wait.
nmhd_status write_ctl_async(nmhd_solver *s, Workspace &w, double time, long long gen, int slot,
                            cudaStream_t stream) {
  StepCtl &h = w.hstage[slot];
  std::memset(&h, 0, sizeof(h));
  h.time = time;
  h.generation = gen;
  h.cfl_cur = h.cfl_next = 0x7f800000u;
  h.goal = INFINITY;
  h.hist_cap = nmhd::kDtHistCap;
  h.dt_seq = w.dt_dev;
  h.dt_seq_base = 0;
  w.parity = 0;
  AD_CUDA(cudaMemcpyAsync(w.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  return NMHD_OK;
}

// One FP32 step with the production kernels on explicit buffers: t.wf holds
// W^n (its margins are filled in place), the raw W^{n+1} goes to t.wo.  The
// kernels take the current state as buffer `parity` of (w0, w1) and the final
// stage flips the device parity; the pair is passed in the order that makes
// t.wf the current buffer, so the parity needs no reset between steps.
// Tensor maps for the buffer set (b0, b1, ws, flux), made on first use (NULL
// where they cannot be made: the kernels then stage by cp.async).
const nmhd::EpilogueMaps *maps_for(nmhd_solver *s, Workspace &w, float *b0, float *b1, float *ws, float *flux) {
  const std::array<const void *, 4> key = {b0, b1, ws, flux};
  auto it = w.maps.find(key);
  if (it != w.maps.end()) return it->second;
  nmhd::EpilogueMaps *m = nmhd::make_epilogue_maps(s->g, b0, b1, ws, flux);
  w.maps[key] = m;
  return m;
}

void prod_step(nmhd_solver *s, Workspace &w, const StepTape<float> &t, bool cfl, cudaStream_t st) {
  const GridParams &g = s->g;
  float *hist = cfl ? w.dt_dev : w.hist_dummy;
  float *b0 = w.parity ? t.wo : t.wf, *b1 = w.parity ? t.wf : t.wo;  // buffer 2 = t.ws
  if (g.my > 0 || g.mz > 0) {
    nmhd::launch_fill(g, w.ctl, b0, b1, st);
    if (cfl) nmhd::launch_cfl_margin(g, w.ctl, b0, b1, st);
  }
  // the default kernels (variant 5), with the tensor maps of this step's
  // buffers (the tape's buffers change from step to step)
  const nmhd::EpilogueMaps *m1 = maps_for(s, w, b0, b1, t.ws, t.f1);
  if (s->cfg.time_order == 1) {
    nmhd::launch_cell_flux_staged(g, w.ctl, b0, b1, t.ws, t.f1, 0, 0, m1, st);
    nmhd::launch_cell_update_fused(g, w.ctl, b0, b1, t.ws, t.f1, hist, 0, 1, 0, 1, m1, st);
  } else {
    const nmhd::EpilogueMaps *m2 = t.f2 == t.f1 ? m1 : maps_for(s, w, b0, b1, t.ws, t.f2);
    nmhd::launch_cell_flux_staged(g, w.ctl, b0, b1, t.ws, t.f1, 0, 1, m1, st);
    nmhd::launch_cell_update_fused(g, w.ctl, b0, b1, t.ws, t.f1, hist, 0, 2, 1, 0, m1, st);
    nmhd::launch_cell_flux_staged(g, w.ctl, b0, b1, t.ws, t.f2, 2, 0, m2, st);
    nmhd::launch_cell_update_fused(g, w.ctl, b0, b1, t.ws, t.f2, hist, 2, 1, 0, 1, m2, st);
  }
  w.parity ^= 1;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// ---------------------------------------------------------------------------
// FP32 (production forward) and FP64 (generic forward) adjoint runs share this
// driver; Prec selects the forward and the real type.
template <class R>
struct Prec;

template <>
struct Prec<float> {
  static constexpr bool kProduction = true;
};
template <>
struct Prec<double> {
  static constexpr bool kProduction = false;
};

template <class R>
nmhd_status run(nmhd_solver *s, int nsteps, int K, const nmhd_loss_spec &L, const float *dt_seq, double *loss_out,
                float *dt_out, R *const grad[8], int grad_on_device, bool want_grad) {
  Workspace &w = workspace(s);
  const size_t n = (size_t)s->g.n;
  const GGrid<R> gg = make_ggrid<R>(s->cfg);
  const int nseg = (nsteps + K - 1) / K;
  const int tape_steps = want_grad ? std::min(K, nsteps) : 1;
  int kseg = 1;  // trailing segments kept on the tape by the forward run
  const bool frozen = dt_seq != nullptr;
  if (!Prec<R>::kProduction && !frozen)
    return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "dt_seq is required for FP64 runs");
  // arena: checkpoints, one segment's tape, the primal pass's ping-pong
  // partner, 3 adjoint states, adjoint scratch, reduction partials
  const size_t nb = (n + 255) / 256;
  R *ckpt = nullptr, *tape = nullptr, *fscr = nullptr, *spare = nullptr, *lam = nullptr, *scr = nullptr;
  R *xslot = nullptr, *fscr2 = nullptr;
  double *partial = nullptr, *acc = nullptr;
  auto carve = [&](Arena &ar) {
    ckpt = want_grad ? ar.take<R>((size_t)nseg * 8 * n) : nullptr;
    tape = ar.take<R>((size_t)kseg * tape_steps * kTapeFields * n);
    // segments recomputed beside the reverse sweep: a second tape slot and a
    // flux scratch of their own
    const bool recompute = want_grad && kseg < nseg;
    xslot = recompute ? ar.take<R>((size_t)tape_steps * kTapeFields * n) : nullptr;
    fscr2 = recompute ? ar.take<R>((size_t)kFluxScratchFields * n) : nullptr;
    fscr = ar.take<R>((size_t)kFluxScratchFields * n);
    spare = ar.take<R>(8 * n);
    lam = want_grad ? ar.take<R>(24 * n) : nullptr;
    scr = want_grad ? ar.take<R>((size_t)kAdjScratchFields * n) : nullptr;
    partial = ar.take<double>(nb);
    acc = ar.take<double>(1);
  };
  Arena probe{0, 0};
  carve(probe);
  if (want_grad && nseg > 1) {
    // more trailing segments on the tape, within the budget
    const size_t seg_bytes = (size_t)tape_steps * kTapeFields * n * sizeof(R);
    long long budget = w.tape_budget;
    if (budget < 0) {
      size_t free_b = 0, total_b = 0;
      AD_CUDA(cudaMemGetInfo(&free_b, &total_b));
      budget = (long long)((free_b + w.bytes) / 2) - (long long)probe.off;
    }
    if (budget > 0) kseg = 1 + (int)std::min<long long>(nseg - 1, budget / (long long)seg_bytes);
    probe = Arena{0, 0};
    carve(probe);
  }
  w.kept_segments = want_grad ? kseg : 0;
  nmhd_status st = reserve(s, w, probe.off + 256);
  if (st != NMHD_OK) return st;
  Arena ar{reinterpret_cast<uintptr_t>(w.mem), 0};
  carve(ar);

  const float *cur;
  double t0;
  st = solver_state(s, &cur, &t0);
  if (st != NMHD_OK) return st;
  cudaStream_t q = s->stream;
  GpuExec ex{q};
  const double scale = stress_scale(s->cfg, L);
  if (frozen) AD_CUDA(cudaMemcpyAsync(w.dt_dev, dt_seq, sizeof(float) * nsteps, cudaMemcpyHostToDevice, q));
  st = write_ctl(s, w, t0, 0, frozen);
  if (st != NMHD_OK) return st;
  AD_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), q));

  // ---- forward run with checkpoints -------------------------------------------
  AD_CUDA(cudaEventRecord(w.ev[0], q));
  StepTape<R> t0tape = tape_at(tape, n, fscr);
  R *A = t0tape.wf, *B = spare;
  if constexpr (Prec<R>::kProduction) {
    AD_CUDA(cudaMemcpyAsync(A, cur, sizeof(float) * 8 * n, cudaMemcpyDeviceToDevice, q));
  } else {
    ex.items((int)(8 * n), OpWiden<R>{cur, nullptr, 0.0, A});
  }
  if (in_window(L, 0)) ex.reduce(gg, OpStress<R, R>{gg, A}, partial, acc, scale);
  std::vector<float> dts(nsteps);
  if (frozen) std::copy(dt_seq, dt_seq + nsteps, dts.begin());
  if constexpr (Prec<R>::kProduction) {
    if (!frozen) {
      // CFL time of the fresh state after its margins are filled (as nmhd_proceed)
      AD_CUDA(cudaMemsetAsync(&w.ctl->parity, 0, sizeof(int), q));
      nmhd::launch_fill(s->g, w.ctl, A, B, q);
      nmhd::launch_cfl_all(s->g, w.ctl, A, B, q);
    }
  }
  std::vector<double> tn(nsteps + 1);
  tn[0] = t0;
  // the last kseg segments' steps are kept on the tape: the reverse sweep
  // runs over them without recomputing them
  const int kept0 = want_grad ? (nseg - kseg) * K : nsteps;
  for (int i = 0; i < nsteps; ++i) {
    if (want_grad && i % K == 0)
      AD_CUDA(cudaMemcpyAsync(ckpt + (size_t)(i / K) * 8 * n, A, sizeof(R) * 8 * n, cudaMemcpyDeviceToDevice, q));
    StepTape<R> t = {A, t0tape.f1, t0tape.ws, t0tape.f2, B};
    if (i >= kept0) {
      t = tape_at(tape + (size_t)(i - kept0) * kTapeFields * n, n, fscr);
      if (t.wf != A) AD_CUDA(cudaMemcpyAsync(t.wf, A, sizeof(R) * 8 * n, cudaMemcpyDeviceToDevice, q));
    }
    if constexpr (Prec<R>::kProduction) {
      prod_step(s, w, t, !frozen, q);
    } else {
      tn[i + 1] = tn[i] + (double)dts[i];
      fwd_step(ex, gg, s->cfg.time_order, tn[i], (R)dts[i], t);
    }
    if (in_window(L, i + 1)) ex.reduce(gg, OpStress<R, R>{gg, t.wo}, partial, acc, scale);
    if (i >= kept0) {
      A = t.wo;
    } else {
      std::swap(A, B);
    }
  }
  AD_CUDA(cudaGetLastError());
  AD_CUDA(cudaEventRecord(w.ev[1], q));
  if constexpr (Prec<R>::kProduction) {
    StepCtl h;
    AD_CUDA(cudaMemcpyAsync(&h, w.ctl, sizeof(h), cudaMemcpyDeviceToHost, q));
    AD_CUDA(cudaStreamSynchronize(q));
    if (h.status)
      return set_err(s, NMHD_ERR_NUMERICAL, "non-finite state, density <= 0 or pressure <= 0 in the forward run");
    if (!frozen) AD_CUDA(cudaMemcpy(dts.data(), w.dt_dev, sizeof(float) * nsteps, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nsteps; ++i) tn[i + 1] = tn[i] + (double)dts[i];
  }
  AD_CUDA(cudaMemcpyAsync(loss_out, acc, sizeof(double), cudaMemcpyDeviceToHost, q));
  AD_CUDA(cudaStreamSynchronize(q));
  if (dt_out) std::copy(dts.begin(), dts.end(), dt_out);
  w.ms[0] = elapsed(w.ev[0], w.ev[1]);
  w.ms[1] = w.ms[2] = 0.0;
  w.ms[3] = w.ms[0];
  if (!want_grad) return NMHD_OK;
  if (Prec<R>::kProduction && !frozen) {
    // the recomputation replays these steps with dt frozen
    AD_CUDA(cudaMemcpyAsync(w.dt_dev, dts.data(), sizeof(float) * nsteps, cudaMemcpyHostToDevice, q));
  }

  // ---- reverse sweep ---------------------------------------------------------------
  // Segments [0, nrec) are recomputed from their checkpoints on a second
  // stream while the reverse sweep runs on a third (high priority): recomputed segment
  // j (from the last, nrec-1, down) lands in slot X for even j and in tape
  // slot 0 for odd j, so the recomputation of a segment overlaps the adjoint
  // of the one after it.  Slot 0 first holds the earliest kept segment; a
  // recomputation into a slot waits for the sweep of its previous segment.
  R *lamA = lam, *lamS = lam + 8 * n, *lamF = lam + 16 * n;
  const AdjScratch<R> sc = scratch_at(scr, n);
  ex.zero(lamA, 8 * n);
  const int nrec = kept0 / K;
  cudaStream_t q2 = w.stream2;
  GpuExec ex2{q2};
  R *slots[2] = {xslot, tape};  // [0] slot X, [1] tape slot 0
  std::vector<cudaEvent_t> rev(2 * (size_t)nrec, nullptr);
  for (auto &e : rev) AD_CUDA(cudaEventCreate(&e));
  auto recompute = [&](int seg) -> nmhd_status {
    const int j = nrec - 1 - seg, si = j % 2;
    const int n0 = seg * K, n1 = std::min(n0 + K, nsteps);
    R *segtape = slots[si];
    AD_CUDA(cudaStreamWaitEvent(q2, w.slot_free[si], 0));
    AD_CUDA(cudaEventRecord(rev[2 * j], q2));
    if constexpr (Prec<R>::kProduction) {
      nmhd_status r = write_ctl_async(s, w, tn[n0], n0, seg, q2);
      if (r != NMHD_OK) return r;
    }
    AD_CUDA(cudaMemcpyAsync(segtape, ckpt + (size_t)seg * 8 * n, sizeof(R) * 8 * n, cudaMemcpyDeviceToDevice, q2));
    for (int i = n0; i < n1; ++i) {
      const StepTape<R> t = tape_at(segtape + (size_t)(i - n0) * kTapeFields * n, n, fscr2);
      if constexpr (Prec<R>::kProduction)
        prod_step(s, w, t, false, q2);
      else
        fwd_step(ex2, gg, s->cfg.time_order, tn[i], (R)dts[i], t);
      if (i + 1 < n1) {
        const StepTape<R> tn1 = tape_at(segtape + (size_t)(i + 1 - n0) * kTapeFields * n, n, fscr2);
        AD_CUDA(cudaMemcpyAsync(tn1.wf, t.wo, sizeof(R) * 8 * n, cudaMemcpyDeviceToDevice, q2));
      }
    }
    AD_CUDA(cudaEventRecord(rev[2 * j + 1], q2));
    AD_CUDA(cudaEventRecord(w.slot_ready[si], q2));
    return NMHD_OK;
  };
  cudaStream_t qs = w.stream_hi;
  GpuExec exs{qs};
  auto sweep = [&](int seg, R *segtape) -> nmhd_status {
    const int n0 = seg * K, n1 = std::min(n0 + K, nsteps);
    for (int i = n1 - 1; i >= n0; --i) {
      const StepTape<R> t = tape_at(segtape + (size_t)(i - n0) * kTapeFields * n, n, fscr);
      if (in_window(L, i + 1)) exs.cells(gg, OpAStress<R>{gg, t.wo, lamA, scale});
      adj_step(exs, gg, s->cfg.time_order, tn[i], (R)dts[i], t, lamA, lamS, lamF, sc);
      std::swap(lamA, lamF);
    }
    return NMHD_OK;
  };
  AD_CUDA(cudaEventRecord(w.ev[2], q));
  // the recomputation and the sweep read the checkpoints, frozen time steps
  // and adjoint state written on q
  AD_CUDA(cudaEventRecord(w.fwd_done, q));
  AD_CUDA(cudaStreamWaitEvent(q2, w.fwd_done, 0));
  AD_CUDA(cudaStreamWaitEvent(qs, w.fwd_done, 0));
  // neither slot holds a segment still to be swept yet
  for (int i = 0; i < 2; ++i) AD_CUDA(cudaEventRecord(w.slot_free[i], qs));
  if (nrec > 0) {
    st = recompute(nrec - 1);
    if (st != NMHD_OK) return st;
  }
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * K;
    if (n0 >= kept0) {  // taped by the forward run
      st = sweep(seg, tape + (size_t)(n0 - kept0) * kTapeFields * n);
      if (st != NMHD_OK) return st;
      if (n0 == kept0) AD_CUDA(cudaEventRecord(w.slot_free[1], qs));  // tape slot 0 swept
      continue;
    }
    const int si = (nrec - 1 - seg) % 2;
    if (seg > 0) {  // the next recomputation overlaps this segment's sweep
      st = recompute(seg - 1);
      if (st != NMHD_OK) return st;
    }
    AD_CUDA(cudaStreamWaitEvent(qs, w.slot_ready[si], 0));
    st = sweep(seg, slots[si]);
    if (st != NMHD_OK) return st;
    AD_CUDA(cudaEventRecord(w.slot_free[si], qs));
  }
  AD_CUDA(cudaGetLastError());
  AD_CUDA(cudaEventRecord(w.sweep_done, qs));
  AD_CUDA(cudaStreamWaitEvent(q, w.sweep_done, 0));
  AD_CUDA(cudaEventRecord(w.ev[3], q));
  AD_CUDA(cudaEventSynchronize(w.ev[3]));
  double ms_re = 0.0;
  for (int j = 0; j < nrec; ++j) ms_re += elapsed(rev[2 * j], rev[2 * j + 1]);
  for (auto &e : rev) cudaEventDestroy(e);
  const double ms_rev = elapsed(w.ev[2], w.ev[3]);
  if (in_window(L, 0)) ex.cells(gg, OpAStress<R>{gg, ckpt, lamA, scale});
  for (int v = 0; v < 8; ++v)
    AD_CUDA(cudaMemcpyAsync(grad[v], lamA + (size_t)v * n, sizeof(R) * n,
                            grad_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, q));
  AD_CUDA(cudaStreamSynchronize(q));
  w.ms[1] = ms_re;
  w.ms[2] = ms_rev;
  w.ms[3] = w.ms[0] + ms_rev;
  return NMHD_OK;
}

}  // namespace

void nmhd_adjoint_release(nmhd_solver *s) {
  if (!s || !s->adjoint) return;
  Workspace *w = static_cast<Workspace *>(s->adjoint);
  if (s->stream) cudaStreamSynchronize(s->stream);
  w->clear_maps();
  cudaFree(w->mem);
  cudaFree(w->ctl);
  cudaFree(w->dt_dev);
  cudaFree(w->hist_dummy);
  for (auto &e : w->ev)
    if (e) cudaEventDestroy(e);
  if (w->stream2) {
    cudaStreamSynchronize(w->stream2);
    cudaStreamDestroy(w->stream2);
  }
  if (w->stream_hi) {
    cudaStreamSynchronize(w->stream_hi);
    cudaStreamDestroy(w->stream_hi);
  }
  if (w->sweep_done) cudaEventDestroy(w->sweep_done);
  if (w->hstage) cudaFreeHost(w->hstage);
  for (int i = 0; i < 2; ++i) {
    if (w->slot_ready[i]) cudaEventDestroy(w->slot_ready[i]);
    if (w->slot_free[i]) cudaEventDestroy(w->slot_free[i]);
  }
  if (w->fwd_done) cudaEventDestroy(w->fwd_done);
  delete w;
  s->adjoint = nullptr;
}

extern "C" {

nmhd_status nmhd_loss_run(nmhd_solver *s, int32_t nsteps, const nmhd_loss_spec *loss, const float *dt_seq,
                          double *loss_out, float *dt_out) {
  nmhd_status st = validate(s, nsteps, 1, loss);
  if (st != NMHD_OK) return st;
  if (!loss_out) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "loss_out is NULL");
  return run<float>(s, nsteps, nsteps, *loss, dt_seq, loss_out, dt_out, nullptr, 0, false);
}

nmhd_status nmhd_adjoint_run(nmhd_solver *s, int32_t nsteps, int32_t ckpt_every, const nmhd_loss_spec *loss,
                             const float *dt_seq, double *loss_out, float *dt_out, float *const grad[8],
                             int on_device) {
  nmhd_status st = validate(s, nsteps, ckpt_every, loss);
  if (st != NMHD_OK) return st;
  if (!loss_out || !grad) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "NULL output");
  for (int v = 0; v < 8; ++v)
    if (!grad[v]) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "grad field pointer is NULL");
  return run<float>(s, nsteps, ckpt_every, *loss, dt_seq, loss_out, dt_out, grad, on_device, true);
}

nmhd_status nmhd_adjoint_run_f64(nmhd_solver *s, int32_t nsteps, int32_t ckpt_every,
                                 const nmhd_loss_spec *loss, const float *dt_seq, double *loss_out,
                                 double *const grad[8]) {
  nmhd_status st = validate(s, nsteps, ckpt_every, loss);
  if (st != NMHD_OK) return st;
  if (!loss_out || !grad || !dt_seq) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  for (int v = 0; v < 8; ++v)
    if (!grad[v]) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "grad field pointer is NULL");
  return run<double>(s, nsteps, ckpt_every, *loss, dt_seq, loss_out, nullptr, grad, 0, true);
}

nmhd_status nmhd_tlm_run(nmhd_solver *s, int32_t nsteps, const nmhd_loss_spec *loss, const float *dt_seq,
                         const double *const dir[8], double shift, double *loss_out, double *dloss_out) {
  nmhd_status st = validate(s, nsteps, 1, loss);
  if (st != NMHD_OK) return st;
  if (!loss_out || !dt_seq) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  typedef Dual<double> D;
  Workspace &w = workspace(s);
  const size_t n = (size_t)s->g.n;
  const size_t nb = (n + 255) / 256;
  D *tape = nullptr, *fscr = nullptr, *spare = nullptr, *partial = nullptr, *acc = nullptr;
  double *dir_dev = nullptr;
  auto carve = [&](Arena &ar) {
    tape = ar.take<D>((size_t)kTapeFields * n);
    fscr = ar.take<D>((size_t)kFluxScratchFields * n);
    spare = ar.take<D>(8 * n);
    dir_dev = ar.take<double>(8 * n);
    partial = ar.take<D>(nb);
    acc = ar.take<D>(1);
  };
  Arena probe{0, 0};
  carve(probe);
  st = reserve(s, w, probe.off + 256);
  if (st != NMHD_OK) return st;
  Arena ar{reinterpret_cast<uintptr_t>(w.mem), 0};
  carve(ar);
  const float *cur;
  double t0;
  st = solver_state(s, &cur, &t0);
  if (st != NMHD_OK) return st;
  cudaStream_t q = s->stream;
  GpuExec ex{q};
  const GGrid<double> gg = make_ggrid<double>(s->cfg);
  const double scale = stress_scale(s->cfg, *loss);
  if (dir)
    for (int v = 0; v < 8; ++v) {
      if (!dir[v]) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "dir field pointer is NULL");
      AD_CUDA(cudaMemcpyAsync(dir_dev + (size_t)v * n, dir[v], sizeof(double) * n, cudaMemcpyHostToDevice, q));
    }
  StepTape<D> t = tape_at(tape, n, fscr);
  D *A = t.wf, *B = spare;
  ex.items((int)(8 * n), OpWiden<D>{cur, dir ? dir_dev : nullptr, shift, A});
  AD_CUDA(cudaMemsetAsync(acc, 0, sizeof(D), q));
  if (in_window(*loss, 0)) ex.reduce(gg, OpStress<D, double>{gg, A}, partial, acc, scale);
  double time = t0;
  for (int i = 0; i < nsteps; ++i) {
    const StepTape<D> ti = {A, t.f1, t.ws, t.f2, B};
    fwd_step(ex, gg, s->cfg.time_order, time, (double)dt_seq[i], ti);
    time = time + (double)dt_seq[i];
    if (in_window(*loss, i + 1)) ex.reduce(gg, OpStress<D, double>{gg, B}, partial, acc, scale);
    std::swap(A, B);
  }
  AD_CUDA(cudaGetLastError());
  D h;
  AD_CUDA(cudaMemcpyAsync(&h, acc, sizeof(D), cudaMemcpyDeviceToHost, q));
  AD_CUDA(cudaStreamSynchronize(q));
  *loss_out = h.v;
  if (dloss_out) *dloss_out = h.d;
  return NMHD_OK;
}

nmhd_status nmhd_adjoint_set_tape_budget(nmhd_solver *s, int64_t bytes) {
  if (!s) return NMHD_ERR_INVALID_ARGUMENT;
  if (bytes < -1) return set_err(s, NMHD_ERR_INVALID_ARGUMENT, "tape budget must be >= -1");
  workspace(s).tape_budget = bytes;
  return NMHD_OK;
}

int32_t nmhd_adjoint_kept_segments(const nmhd_solver *s) {
  if (!s || !s->adjoint) return 0;
  return static_cast<const Workspace *>(s->adjoint)->kept_segments;
}

nmhd_status nmhd_adjoint_timing(const nmhd_solver *s, double ms_out[4]) {
  if (!s || !ms_out) return NMHD_ERR_INVALID_ARGUMENT;
  if (!s->adjoint) {
    for (int i = 0; i < 4; ++i) ms_out[i] = 0.0;
    return NMHD_OK;
  }
  const Workspace *w = static_cast<const Workspace *>(s->adjoint);
  for (int i = 0; i < 4; ++i) ms_out[i] = w->ms[i];
  return NMHD_OK;
}

}  // extern "C"
