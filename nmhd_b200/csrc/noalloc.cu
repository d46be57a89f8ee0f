// Allocation-free entry point: nmhd_advance_noalloc (include/nmhd.h).
//
// Some callers cannot call cudaMalloc: a host framework whose caching
// allocator has reserved the device memory (an allocation of ours would fail
// or fragment its pool), or a real-time loop where a device allocation and the
// implicit device synchronisation it can bring are not allowed.  For them this
// file keeps all the scratch of the tiled time step in one static __device__
// array and advances a caller-owned state without allocating anything.
//
// The array below is part of this library's device image: every GPU that
// loads the library holds it (kNoAllocScratchFloats floats, about 28 MB)
// until the process exits.  All calls share it and it keeps the last call's
// contents, so calls that overlap on the GPU race; the control block at its
// start is rewritten by every call.  The first call on a device does the
// set-up (the array's device address, looked up with that device current);
// it should come before any stream capture.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <string>

#include "../../include/nmhd.h"
#include "step.cuh"

namespace {

// Largest box (cells including margins) the allocation-free path accepts.
constexpr long long kNoAllocMaxCells = NMHD_NOALLOC_MAX_CELLS;
// Control block + dt history, then 27 fields of kNoAllocMaxCells floats:
// second state buffer (8), predictor (8), conserved update (5), B fluxes (6).
constexpr size_t kCtlFloats = 256;  // sizeof(StepCtl) rounded up, in floats
constexpr size_t kNoAllocScratchFloats =
    kCtlFloats + nmhd::kDtHistCap + 27 * (size_t)kNoAllocMaxCells;
// Steps enqueued between two reads of the control block (the call stops
// early once the goal is reached or the state goes bad).
constexpr int64_t kStepsPerCheck = 16;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

thread_local std::string g_noalloc_error;
// Device address of the array, per device.  Host threads may make their first
// call on a device at the same time: each looks the address up (the same
// value) and stores it atomically.
constexpr int kMaxDevices = 64;
std::atomic<float *> g_scratch_ptr[kMaxDevices];

nmhd_status noalloc_fail(nmhd_status st, const std::string &msg) {
  g_noalloc_error = msg;
  return st;
}

}  // namespace

extern "C" const char *nmhd_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

extern "C" nmhd_status nmhd_advance_noalloc(const nmhd_config *cfg, const float *state_in,
                                            float *state_out, double *time, int64_t *generation,
                                            double goal_time, int64_t nsteps, int64_t *steps_done,
                                            void *cuda_stream) {
  static_assert(sizeof(nmhd::StepCtl) <= kCtlFloats * sizeof(float), "control block too large");
  if (steps_done) *steps_done = 0;
  if (!cfg || !state_in || !state_out || !time || !generation || nsteps < 0)
    return noalloc_fail(NMHD_ERR_INVALID_ARGUMENT, "NULL argument or negative nsteps");
  if (state_in == state_out)
    return noalloc_fail(NMHD_ERR_INVALID_ARGUMENT, "state_in and state_out must not alias");
  // nmhd_create's rules, then the whole-box rules of this path
  std::string why;
  const nmhd_status vs = nmhd::validate_config(cfg, why);
  if (vs != NMHD_OK) return noalloc_fail(vs, why);
  if (cfg->parallel_size_y > 1 || cfg->flags != 0)
    return noalloc_fail(NMHD_ERR_INVALID_ARGUMENT,
                        "invalid configuration (a whole box: parallel_size_y <= 1, flags 0)");
  const long long cells = (long long)cfg->size_x * cfg->size_y * cfg->size_z;
  if (cells > kNoAllocMaxCells)
    return noalloc_fail(NMHD_ERR_INVALID_ARGUMENT,
                        "box has " + std::to_string(cells) + " cells; the allocation-free path holds at most " +
                            std::to_string(kNoAllocMaxCells));
  // An error left by earlier work on this thread is not this call's: report
  // it without consuming it, and launch nothing.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return noalloc_fail(NMHD_ERR_CUDA, std::string("a CUDA error from earlier work is pending: ") +
                                           cudaGetErrorString(e));
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(NMHD_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(NMHD_ERR_NOT_SUPPORTED, "device index >= 64");
  // Set-up, once per device with that device current: the host-side name of a
  // __device__ array is not a device address; ask the runtime for it.
  float *base = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!base) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return noalloc_fail(NMHD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    base = static_cast<float *>(p);
    g_scratch_ptr[dev].store(base, std::memory_order_release);
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const size_t n = (size_t)cells;
  nmhd::StepCtl *ctl = reinterpret_cast<nmhd::StepCtl *>(base);
  float *dt_hist = base + kCtlFloats;
  float *w1 = dt_hist + nmhd::kDtHistCap;
  float *wp = w1 + 8 * n;
  float *unew = wp + 8 * n;
  float *bflux = unew + 5 * n;
  float *w0 = state_out;

  nmhd::GridParams g = nmhd::derive_grid(*cfg);
  // Control block: everything that must start at zero starts at zero.
  nmhd::StepCtl h;
  std::memset(&h, 0, sizeof(h));
  h.time = *time;
  h.generation = *generation;
  h.cfl_cur = h.cfl_next = 0x7f800000u;
  h.goal = (float)goal_time;
  h.hist_cap = nmhd::kDtHistCap;
  e = cudaMemcpyAsync(ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(w0, state_in, sizeof(float) * 8 * n, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return noalloc_fail(NMHD_ERR_CUDA, cudaGetErrorString(e));
  const nmhd::TileShape shape = {8, 16};
  nmhd::launch_fill(g, ctl, w0, w1, st);
  nmhd::launch_cfl_all(g, ctl, w0, w1, st);
  // Steps in groups of kStepsPerCheck; after each group the control block is
  // read back and the call stops once the goal is reached or the state is bad
  // (steps enqueued past that point return at once on the device).
  for (int64_t done = 0; done < nsteps;) {
    const int64_t group = nsteps - done < kStepsPerCheck ? nsteps - done : kStepsPerCheck;
    for (int64_t i = 0; i < group; ++i) {
      if (g.my > 0 || g.mz > 0) {
        nmhd::launch_fill(g, ctl, w0, w1, st);
        nmhd::launch_cfl_margin(g, ctl, w0, w1, st);
      }
      if (cfg->time_order == 1) {
        nmhd::launch_tile_stage(g, ctl, w0, w1, wp, unew, bflux, dt_hist, 0, 1, 0, 1, shape, st);
      } else {
        nmhd::launch_tile_stage(g, ctl, w0, w1, wp, unew, bflux, dt_hist, 0, 2, 1, 0, shape, st);
        nmhd::launch_tile_stage(g, ctl, w0, w1, wp, unew, bflux, dt_hist, 2, 1, 0, 1, shape, st);
      }
    }
    done += group;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(NMHD_ERR_CUDA, cudaGetErrorString(e));
    if (h.done || h.status) break;
  }
  if (nsteps == 0) {
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(NMHD_ERR_CUDA, cudaGetErrorString(e));
  }
  // The result is in the current buffer; bring it to state_out if it ended in scratch.
  if (h.parity == 1) {
    e = cudaMemcpyAsync(state_out, w1, sizeof(float) * 8 * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(NMHD_ERR_CUDA, cudaGetErrorString(e));
  }
  if (steps_done) *steps_done = h.generation - *generation;
  *time = h.time;
  *generation = h.generation;
  if (h.status)
    return noalloc_fail(NMHD_ERR_NUMERICAL, "non-finite state, density <= 0, pressure <= 0 or bad dt");
  return h.done ? NMHD_GOAL_REACHED : NMHD_STEP_LIMIT;
}
