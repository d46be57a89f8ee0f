// C ABI of the B200-native ideal-MHD solver: the host side of MHDSolver
// (src/library/mhd_solver.hrb:150-276, mhd_solver.inlrb:69-97, 850-1050).
//
// One nmhd_solver owns the device state of one box: two primitive-state
// buffers (current / next, swapped on the device every step), the RK
// predictor, the face-flux scratch and a device-resident step control block.
// proceed() enqueues whole steps without any host round trip; batches of
// steps are captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/nmhd.h"
#include "solver_impl.h"
#include "step.cuh"

using nmhd::GridParams;
using nmhd::StepCtl;

namespace {

const char *kVersion = "nmhd_b200 0.1 (sm_100a)";
thread_local std::string g_create_error;

nmhd_status fail(nmhd_solver *s, nmhd_status st, const std::string &msg) {
  if (s) s->err = msg;
  else g_create_error = msg;
  return st;
}

nmhd_status cuda_fail(nmhd_solver *s, cudaError_t e, const char *what) {
  return fail(s, e == cudaErrorMemoryAllocation ? NMHD_ERR_OUT_OF_MEMORY : NMHD_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define NMHD_CUDA(s, call)                                \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(s, e_, #call); \
  } while (0)

}  // namespace

// Derived constants exactly as the reference's float chains produce them
// (simulation_config_default.h:56-103; relative_velocity of
// src/application/kepler_disk_demo/mhd_solver.curb:50-52).
GridParams nmhd::derive_grid(const nmhd_config &c) {
  GridParams g;
  g.sx = c.size_x;
  g.sy = c.size_y;
  g.sz = c.size_z;
  g.n = c.size_x * c.size_y * c.size_z;
  g.my = c.margin_y;
  g.mz = c.margin_z;
  // A radial slab of a box split over P ranks along Y: kGlobalSizeY = P * the
  // slab's interior rows, extent_y is the whole box's (kGlobalExtentY).
  const int py = c.parallel_size_y > 1 ? c.parallel_size_y : 1;
  const int s[3] = {c.size_x, c.size_y, c.size_z};
  const int li[3] = {c.size_x, c.size_y - 2 * c.margin_y, c.size_z - 2 * c.margin_z};
  const int gi[3] = {li[0], py * li[1], li[2]};
  const float L[3] = {c.extent_x, c.extent_y, c.extent_z};
  volatile float comp[3], local[3], d[3];
  for (int i = 0; i < 3; ++i) {
    volatile float per = L[i] / (float)gi[i];
    comp[i] = per * (float)s[i];
    local[i] = per * (float)li[i];
    d[i] = comp[i] / (float)s[i];
  }
  g.dx = d[0];
  g.dy = d[1];
  g.dz = d[2];
  g.extent_x = comp[0];
  g.corner_y = -comp[1] / 2.0f;
  g.gamma = c.gamma;
  g.cfl = c.cfl;
  g.q = c.q;
  g.omega = c.omega;
  volatile float qo = -c.q * c.omega;
  volatile float rv = qo * local[1];
  g.shear = c.problem == NMHD_PROBLEM_SHEARING_BOX;
  // relative_velocity() hook: zero without a shearing box
  g.rel_vel = g.shear ? (double)rv : 0.0;
  g.order2 = c.space_order != 1;
  auto pow2 = [](float v) {
    int e;
    return v > 0.0f && std::isfinite(v) && std::frexp(v, &e) == 0.5f && e > -125 && e < 126;
  };
  g.pow2_spacing = pow2(g.dx) && pow2(g.dy) && pow2(g.dz);
  g.inv_dx = 1.0f / g.dx;
  g.inv_dy = 1.0f / g.dy;
  g.inv_dz = 1.0f / g.dz;
  return g;
}

nmhd_status nmhd::validate_config(const nmhd_config *c, std::string &why) {
  if (!c) { why = "config is NULL"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->size_x < 1 || c->size_y < 1 || c->size_z < 1) { why = "sizes must be >= 1"; return NMHD_ERR_INVALID_ARGUMENT; }
  const long long n = (long long)c->size_x * c->size_y * c->size_z;
  if (n * 8 >= (1LL << 31)) { why = "box too large: 8*cells must fit in int32"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->margin_y < 0 || c->margin_z < 0) { why = "margins must be >= 0"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->size_y - 2 * c->margin_y < c->margin_y || (c->margin_y > 0 && c->size_y - 2 * c->margin_y < 1)) {
    why = "interior Y rows must be at least margin_y"; return NMHD_ERR_INVALID_ARGUMENT;
  }
  if (c->margin_z > 0 && c->size_z - 2 * c->margin_z < c->margin_z) {
    why = "interior Z planes must be at least margin_z"; return NMHD_ERR_INVALID_ARGUMENT;
  }
  if (!(c->extent_x > 0 && c->extent_y > 0 && c->extent_z > 0)) { why = "extents must be > 0"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (!(c->gamma > 1.0f) || !(c->cfl > 0.0f)) { why = "gamma must be > 1 and cfl > 0"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->problem != NMHD_PROBLEM_NONE && c->problem != NMHD_PROBLEM_SHEARING_BOX) { why = "unknown problem"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->space_order != 1 && c->space_order != 2) { why = "space_order must be 1 or 2"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->time_order != 1 && c->time_order != 2) { why = "time_order must be 1 or 2"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->parallel_size_y < 0) { why = "parallel_size_y must be >= 0"; return NMHD_ERR_INVALID_ARGUMENT; }
  if (c->flags & ~(NMHD_FLAG_HALO_PER_STAGE | NMHD_FLAG_FAST_ARITHMETIC)) {
    why = "unknown flags"; return NMHD_ERR_INVALID_ARGUMENT;
  }
  if ((c->flags & NMHD_FLAG_HALO_PER_STAGE) && c->parallel_size_y > 1) {
    why = "per-stage margin fill is for whole boxes"; return NMHD_ERR_NOT_SUPPORTED;
  }
  if (c->parallel_size_y > 1 && c->margin_y < 1) {
    why = "a radial slab (parallel_size_y > 1) needs margin_y >= 1"; return NMHD_ERR_INVALID_ARGUMENT;
  }
  return NMHD_OK;
}

namespace {

nmhd_status read_ctl(nmhd_solver *s, StepCtl &h) {
  NMHD_CUDA(s, cudaMemcpyAsync(&h, s->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s->stream));
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  return NMHD_OK;
}

nmhd_status write_ctl(nmhd_solver *s, const StepCtl &h) {
  NMHD_CUDA(s, cudaMemcpyAsync(s->ctl, &h, sizeof(StepCtl), cudaMemcpyHostToDevice, s->stream));
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  return NMHD_OK;
}

float *current_buffer(nmhd_solver *s, const StepCtl &h) { return h.parity ? s->w1 : s->w0; }

// Steps per CUDA graph of nmhd_proceed.
constexpr int kStepBatch = 16;

// One RK stage with the selected kernel variant.
void enqueue_stage(nmhd_solver *s, int in_sel, int out_sel, int half, int final_stage, cudaStream_t st) {
  const GridParams &g = s->g;
  if (s->variant == 0) {
    float *unew = s->flux, *bflux = s->flux + (size_t)5 * g.n;
    nmhd::launch_tile_stage(g, s->ctl, s->w0, s->w1, s->wp, unew, bflux, s->dt_hist, in_sel, out_sel,
                            half, final_stage, s->shape, st);
  } else if (s->variant == 2 || s->variant == 4 || s->variant == 5) {
    if (s->cfg.flags & NMHD_FLAG_FAST_ARITHMETIC)
      nmhd::launch_cell_flux_fast(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, s->epi_maps, st);
    else if (s->variant == 5)
      nmhd::launch_cell_flux_staged(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, s->epi_maps, st);
    else
      nmhd::launch_cell_flux(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, st);
    if (s->variant == 4 || s->variant == 5)
      nmhd::launch_cell_update_fused(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel, half,
                                     final_stage, s->epi_maps, st);
    else
      nmhd::launch_cell_update(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel, half,
                               final_stage, st);
  } else if (s->variant == 3) {
    nmhd::launch_cell_stage_chunked(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel, half,
                                    final_stage, s->shape.zc, st);
  } else {
    nmhd::launch_stage(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel, half,
                       final_stage, st);
  }
}

// One time step, enqueued on the solver's stream (mhd_solver.inlrb:865-985).
void enqueue_step(nmhd_solver *s) {
  const GridParams &g = s->g;
  cudaStream_t st = s->stream;
  if (g.my > 0 || g.mz > 0) {
    nmhd::launch_fill(g, s->ctl, s->w0, s->w1, st);
    nmhd::launch_cfl_margin(g, s->ctl, s->w0, s->w1, st);
  }
  if (s->cfg.time_order == 1) {
    enqueue_stage(s, 0, 1, 0, 1, st);
  } else {
    enqueue_stage(s, 0, 2, 1, 0, st);
    if (s->cfg.flags & NMHD_FLAG_HALO_PER_STAGE) nmhd::launch_fill_predictor(g, s->ctl, s->wp, st);
    enqueue_stage(s, 2, 1, 0, 1, st);
  }
}

nmhd_status graph_for(nmhd_solver *s, int steps, cudaGraphExec_t *out) {
  auto it = s->graphs.find(steps);
  if (it != s->graphs.end()) { *out = it->second; return NMHD_OK; }
  cudaGraph_t graph;
  NMHD_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < steps; ++i) enqueue_step(s);
  NMHD_CUDA(s, cudaStreamEndCapture(s->stream, &graph));
  cudaGraphExec_t exec;
  cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaGraphInstantiate");
  s->graphs[steps] = exec;
  // upload now, so that the first launch does not pay for it
  NMHD_CUDA(s, cudaGraphUpload(exec, s->stream));
  *out = exec;
  return NMHD_OK;
}

void drop_graphs(nmhd_solver *s) {
  for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
}

nmhd_status copy_fields(nmhd_solver *s, float *dev_base, const float *const in[8], float *const out[8],
                        int on_device) {
  const size_t bytes = sizeof(float) * (size_t)s->g.n;
  for (int v = 0; v < 8; ++v) {
    if (in) {
      if (!in[v]) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "field pointer is NULL");
      NMHD_CUDA(s, cudaMemcpyAsync(dev_base + (size_t)v * s->g.n, in[v], bytes,
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->stream));
    } else {
      if (!out[v]) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "field pointer is NULL");
      NMHD_CUDA(s, cudaMemcpyAsync(out[v], dev_base + (size_t)v * s->g.n, bytes,
                                   on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s->stream));
    }
  }
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  return NMHD_OK;
}

}  // namespace

// Kernel choice of nmhd_autotune for boxes of this shape, if one was tuned
// in this process (defined with the autotuner below).
void apply_tuned(nmhd_solver *s);

extern "C" {

const char *nmhd_version(void) { return kVersion; }

nmhd_status nmhd_create(const nmhd_config *cfg, nmhd_solver **out) {
  if (!out) return fail(nullptr, NMHD_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  std::string why;
  nmhd_status st = nmhd::validate_config(cfg, why);
  if (st != NMHD_OK) return fail(nullptr, st, why);
  nmhd_solver *s = new nmhd_solver();
  s->cfg = *cfg;
  s->g = nmhd::derive_grid(*cfg);
  cudaError_t e = cudaGetDevice(&s->device);
  const size_t n = (size_t)s->g.n;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) s->own_stream = true;
  if (e == cudaSuccess) e = cudaMalloc(&s->w0, sizeof(float) * 8 * n);
  if (e == cudaSuccess) e = cudaMalloc(&s->w1, sizeof(float) * 8 * n);
  if (e == cudaSuccess) e = cudaMalloc(&s->wp, sizeof(float) * 8 * n);
  if (e == cudaSuccess) e = cudaMalloc(&s->flux, sizeof(float) * nmhd::kFluxFields * n);
  if (e == cudaSuccess) e = cudaMalloc(&s->dt_hist, sizeof(float) * nmhd::kDtHistCap);
  if (e == cudaSuccess) e = cudaMalloc(&s->ctl, sizeof(StepCtl));
  if (e == cudaSuccess) e = cudaMalloc(&s->diag, sizeof(double) * nmhd::kDiagFields);
  if (e == cudaSuccess) e = cudaMallocHost(&s->hctl, 2 * sizeof(StepCtl));
  for (int i = 0; i < 2 && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&s->batch_done[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->w0, 0, sizeof(float) * 8 * n, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->w1, 0, sizeof(float) * 8 * n, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->wp, 0, sizeof(float) * 8 * n, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->dt_hist, 0, sizeof(float) * nmhd::kDtHistCap, s->stream);
  if (e != cudaSuccess) {
    nmhd_status r = cuda_fail(nullptr, e, "nmhd_create");
    nmhd_destroy(s);
    return r;
  }
  StepCtl h;
  std::memset(&h, 0, sizeof(h));
  h.cfl_cur = h.cfl_next = 0x7f800000u;
  h.goal = INFINITY;
  h.hist_cap = nmhd::kDtHistCap;
  st = write_ctl(s, h);
  if (st != NMHD_OK) {
    g_create_error = s->err;
    nmhd_destroy(s);
    return st;
  }
  s->epi_maps = nmhd::make_epilogue_maps(s->g, s->w0, s->w1, s->wp, s->flux);
  apply_tuned(s);
  *out = s;
  return NMHD_OK;
}

void nmhd_destroy(nmhd_solver *s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  nmhd_adjoint_release(s);
  nmhd::free_epilogue_maps(s->epi_maps);
  cudaFree(s->w0);
  cudaFree(s->w1);
  cudaFree(s->wp);
  cudaFree(s->flux);
  cudaFree(s->dt_hist);
  cudaFree(s->ctl);
  cudaFree(s->diag);
  if (s->hctl) cudaFreeHost(s->hctl);
  for (cudaEvent_t ev : s->batch_done)
    if (ev) cudaEventDestroy(ev);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

nmhd_status nmhd_set_state(nmhd_solver *s, const float *const fields[8], int on_device) {
  if (!s || !fields) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  st = copy_fields(s, current_buffer(s, h), fields, nullptr, on_device);
  if (st != NMHD_OK) return st;
  // A new state: its CFL time must be recomputed and earlier errors no longer apply.
  h.status = 0;
  h.done = 0;
  h.cfl_cur = h.cfl_next = 0x7f800000u;
  s->cfl_ready = false;
  return write_ctl(s, h);
}

nmhd_status nmhd_get_state(nmhd_solver *s, float *const fields[8], int on_device) {
  if (!s || !fields) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  return copy_fields(s, current_buffer(s, h), nullptr, fields, on_device);
}

nmhd_status nmhd_read(nmhd_solver *s, const char *path) {
  if (!s || !path) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return fail(s, NMHD_ERR_IO, std::string("cannot open ") + path);
  int32_t sz[3];
  if (std::fread(sz, sizeof(int32_t), 3, fp) != 3) {
    std::fclose(fp);
    return fail(s, NMHD_ERR_IO, std::string("truncated header in ") + path);
  }
  if (sz[0] != s->g.sx || sz[1] != s->g.sy || sz[2] != s->g.sz) {
    std::fclose(fp);
    char buf[160];
    std::snprintf(buf, sizeof buf, "size mismatch: file %dx%dx%d, solver %dx%dx%d", sz[0], sz[1], sz[2],
                  s->g.sx, s->g.sy, s->g.sz);
    return fail(s, NMHD_ERR_SIZE_MISMATCH, buf);
  }
  const size_t n = (size_t)s->g.n;
  std::vector<float> host(8 * n);
  const size_t got = std::fread(host.data(), sizeof(float), 8 * n, fp);
  std::fclose(fp);
  if (got != 8 * n) return fail(s, NMHD_ERR_IO, std::string("truncated data in ") + path);
  const float *f[8];
  for (int v = 0; v < 8; ++v) f[v] = host.data() + v * n;
  return nmhd_set_state(s, f, 0);
}

nmhd_status nmhd_write(nmhd_solver *s, const char *path) {
  if (!s || !path) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  const size_t n = (size_t)s->g.n;
  std::vector<float> host(8 * n);
  float *f[8];
  for (int v = 0; v < 8; ++v) f[v] = host.data() + v * n;
  nmhd_status st = nmhd_get_state(s, f, 0);
  if (st != NMHD_OK) return st;
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return fail(s, NMHD_ERR_IO, std::string("cannot open ") + path);
  const int32_t sz[3] = {s->g.sx, s->g.sy, s->g.sz};
  bool ok = std::fwrite(sz, sizeof(int32_t), 3, fp) == 3;
  ok = ok && std::fwrite(host.data(), sizeof(float), 8 * n, fp) == 8 * n;
  ok = (std::fclose(fp) == 0) && ok;
  return ok ? NMHD_OK : fail(s, NMHD_ERR_IO, std::string("cannot write ") + path);
}

nmhd_status nmhd_proceed(nmhd_solver *s, double goal_time, double wallclock_limit, int64_t max_steps,
                         int64_t *steps_done) {
  if (steps_done) *steps_done = 0;
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  if (s->cfg.parallel_size_y > 1)
    return fail(s, NMHD_ERR_NOT_SUPPORTED, "a radial slab steps through nmhd_halo_pack/unpack and nmhd_step_stages");
  const auto t0 = std::chrono::steady_clock::now();
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  if (h.status) return fail(s, NMHD_ERR_NUMERICAL, "state is not valid (set a new state)");
  const long long gen0 = h.generation;
  h.goal = (float)goal_time;
  h.done = 0;
  if (!s->cfl_ready) {
    h.cfl_cur = h.cfl_next = 0x7f800000u;
    h.blocks_done = 0;
  }
  st = write_ctl(s, h);
  if (st != NMHD_OK) return st;
  if (!s->cfl_ready) {
    // CFL time of the fresh state, after its margins are filled.
    nmhd::launch_fill(s->g, s->ctl, s->w0, s->w1, s->stream);
    nmhd::launch_cfl_all(s->g, s->ctl, s->w0, s->w1, s->stream);
    NMHD_CUDA(s, cudaGetLastError());
    s->cfl_ready = true;
  }
  // Batches of kStepBatch steps, each one CUDA graph followed by a copy of the
  // control block to pinned host memory.  Without a wallclock limit the next
  // batch is launched before the previous one's control block is read, so the
  // GPU does not idle while the host checks it; a batch launched after the
  // goal step returns at once on the device (every kernel tests `done`).
  // With a wallclock limit one batch at a time is in flight, so the limit
  // stops the run within one batch, as before.
  long long left = max_steps > 0 ? max_steps : -1;
  const int depth = wallclock_limit > 0 ? 1 : 2;
  int queue[2], queued = 0, head = 0, next_slot = 0;
  nmhd_status result = NMHD_OK;
  for (;;) {
    while (queued < depth && left != 0) {
      int batch = kStepBatch;
      if (left >= 0 && left < batch) batch = (int)left;
      cudaGraphExec_t ge;
      st = graph_for(s, batch, &ge);
      if (st != NMHD_OK) return st;
      const int slot = next_slot;
      next_slot ^= 1;
      NMHD_CUDA(s, cudaGraphLaunch(ge, s->stream));
      NMHD_CUDA(s, cudaMemcpyAsync(&s->hctl[slot], s->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s->stream));
      NMHD_CUDA(s, cudaEventRecord(s->batch_done[slot], s->stream));
      queue[(head + queued) % 2] = slot;
      ++queued;
      if (left > 0) left -= batch;
    }
    if (queued == 0) { result = NMHD_STEP_LIMIT; break; }
    const int slot = queue[head];
    head = (head + 1) % 2;
    --queued;
    NMHD_CUDA(s, cudaEventSynchronize(s->batch_done[slot]));
    h = s->hctl[slot];
    if (h.status) {
      result = fail(s, NMHD_ERR_NUMERICAL,
                    (h.status & nmhd::kStatusTimeout) ? "a kernel's bounded wait for its tensor copies gave up"
                    : (h.status & nmhd::kStatusBadDt) ? "time step is negative or not finite"
                                                      : "non-finite state, density <= 0 or pressure <= 0");
      break;
    }
    if (h.done) { result = NMHD_GOAL_REACHED; break; }
    if (wallclock_limit > 0) {
      const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > wallclock_limit) { result = NMHD_TIMEOUT; break; }
    }
  }
  // a batch still in flight ran after the goal or the error: its kernels
  // returned at once and the clock read above is final
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  if (steps_done) *steps_done = h.generation - gen0;
  return result;
}

nmhd_status nmhd_prepare(nmhd_solver *s, int64_t max_steps) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  if (s->cfg.parallel_size_y > 1)
    return fail(s, NMHD_ERR_NOT_SUPPORTED, "a radial slab steps through nmhd_halo_pack/unpack and nmhd_step_stages");
  cudaGraphExec_t ge;
  const int first = max_steps > 0 && max_steps < kStepBatch ? (int)max_steps : kStepBatch;
  nmhd_status st = graph_for(s, first, &ge);
  if (st == NMHD_OK && max_steps > kStepBatch && max_steps % kStepBatch)
    st = graph_for(s, (int)(max_steps % kStepBatch), &ge);
  return st;
}

double nmhd_current_time(const nmhd_solver *s) {
  if (!s) return NAN;
  StepCtl h;
  if (read_ctl(const_cast<nmhd_solver *>(s), h) != NMHD_OK) return NAN;
  return h.time;
}

int64_t nmhd_generation(const nmhd_solver *s) {
  if (!s) return -1;
  StepCtl h;
  if (read_ctl(const_cast<nmhd_solver *>(s), h) != NMHD_OK) return -1;
  return h.generation;
}

nmhd_status nmhd_set_time(nmhd_solver *s, double current_time, int64_t generation) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  h.time = current_time;
  h.generation = generation;
  // The shearing fill depends on the time: recompute margins and CFL.
  s->cfl_ready = false;
  return write_ctl(s, h);
}

int64_t nmhd_dt_history(const nmhd_solver *s, float *out, int64_t n) {
  if (!s || !out || n <= 0) return 0;
  nmhd_solver *m = const_cast<nmhd_solver *>(s);
  StepCtl h;
  if (read_ctl(m, h) != NMHD_OK) return 0;
  std::vector<float> all(nmhd::kDtHistCap);
  if (cudaMemcpy(all.data(), s->dt_hist, sizeof(float) * nmhd::kDtHistCap, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return 0;
  long long avail = h.generation < nmhd::kDtHistCap ? h.generation : nmhd::kDtHistCap;
  long long k = n < avail ? n : avail;
  for (long long i = 0; i < k; ++i) {
    long long gen = h.generation - k + i;
    out[i] = all[gen % nmhd::kDtHistCap];
  }
  return k;
}

nmhd_status nmhd_diagnostics(nmhd_solver *s, nmhd_diag *out) {
  if (!s || !out) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL argument");
  NMHD_CUDA(s, cudaMemsetAsync(s->diag, 0, sizeof(double) * nmhd::kDiagFields, s->stream));
  nmhd::launch_diag(s->g, s->ctl, s->w0, s->w1, s->diag, s->stream);
  NMHD_CUDA(s, cudaGetLastError());
  double a[nmhd::kDiagFields];
  NMHD_CUDA(s, cudaMemcpyAsync(a, s->diag, sizeof(a), cudaMemcpyDeviceToHost, s->stream));
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  std::memset(out, 0, sizeof(*out));
  out->mass = a[0];
  out->momentum[0] = a[1];
  out->momentum[1] = a[2];
  out->momentum[2] = a[3];
  out->kinetic_energy = a[4];
  out->internal_energy = a[5];
  out->magnetic_energy = a[6];
  out->total_energy = a[4] + a[5] + a[6];
  out->volume = a[8];
  out->maxwell_stress = a[8] > 0 ? a[7] / a[8] : 0.0;
  out->bx2_mean = a[9] / (double)s->g.n;
  out->by2_mean = a[10] / (double)s->g.n;
  out->max_div_b = a[nmhd::kDiagFields - 1];
  return NMHD_OK;
}

namespace {
const char *kKernelNames[] = {"fill_margins", "cfl_margins", "flux_stage1", "update_stage1",
                              "flux_stage2", "update_stage2"};
constexpr int kKernelClasses = 6;
}  // namespace

const char *nmhd_kernel_name(int i) {
  return (i >= 0 && i < kKernelClasses) ? kKernelNames[i] : nullptr;
}

int nmhd_profile(nmhd_solver *s, int steps, double *ms_out, double *launches_out, int max) {
  if (!s || !ms_out || steps <= 0 || max <= 0) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  if (s->cfg.parallel_size_y > 1)
    return fail(s, NMHD_ERR_NOT_SUPPORTED, "a radial slab steps through nmhd_halo_pack/unpack and nmhd_step_stages");
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  h.goal = INFINITY;
  h.done = 0;
  if (!s->cfl_ready) h.cfl_cur = h.cfl_next = 0x7f800000u;
  st = write_ctl(s, h);
  if (st != NMHD_OK) return st;
  if (!s->cfl_ready) {
    nmhd::launch_fill(s->g, s->ctl, s->w0, s->w1, s->stream);
    nmhd::launch_cfl_all(s->g, s->ctl, s->w0, s->w1, s->stream);
    s->cfl_ready = true;
  }
  cudaEvent_t ev[kKernelClasses + 1];
  for (auto &e : ev) NMHD_CUDA(s, cudaEventCreate(&e));
  double acc[kKernelClasses] = {0};
  double cnt[kKernelClasses] = {0};
  const GridParams &g = s->g;
  cudaStream_t q = s->stream;
  const bool margins = g.my > 0 || g.mz > 0;
  const bool midpoint = s->cfg.time_order != 1;
  for (int it = 0; it < steps; ++it) {
    NMHD_CUDA(s, cudaEventRecord(ev[0], q));
    if (margins) nmhd::launch_fill(g, s->ctl, s->w0, s->w1, q);
    NMHD_CUDA(s, cudaEventRecord(ev[1], q));
    if (margins) nmhd::launch_cfl_margin(g, s->ctl, s->w0, s->w1, q);
    NMHD_CUDA(s, cudaEventRecord(ev[2], q));
    float *unew = s->flux, *bflux = s->flux + (size_t)5 * g.n;
    // each stage as its two kernels (flux, then update / CT), separately timed
    // variant 3 interleaves the two kernels by chunk: its whole stage is
    // timed in the flux class and the update class reads 0
    auto flux_k = [&](int in_sel, int half) {
      if (s->variant == 3) return;
      if (s->variant == 0)
        nmhd::launch_tile_flux(g, s->ctl, s->w0, s->w1, s->wp, unew, bflux, in_sel, half, s->shape, q);
      else if ((s->variant == 2 || s->variant == 4 || s->variant == 5) && (s->cfg.flags & NMHD_FLAG_FAST_ARITHMETIC))
        nmhd::launch_cell_flux_fast(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, s->epi_maps, q);
      else if (s->variant == 5)
        nmhd::launch_cell_flux_staged(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, s->epi_maps, q);
      else if (s->variant == 2 || s->variant == 4)
        nmhd::launch_cell_flux(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, q);
      else
        nmhd::launch_flux(g, s->ctl, s->w0, s->w1, s->wp, s->flux, in_sel, half, q);
    };
    auto upd_k = [&](int in_sel, int out_sel, int half, int fin) {
      if (s->variant == 3) return;
      if (s->variant == 0)
        nmhd::launch_tile_ct(g, s->ctl, s->w0, s->w1, s->wp, unew, bflux, s->dt_hist, in_sel, out_sel,
                             half, fin, s->shape, q);
      else if (s->variant == 2)
        nmhd::launch_cell_update(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel,
                                 half, fin, q);
      else if (s->variant == 4 || s->variant == 5)
        nmhd::launch_cell_update_fused(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel,
                                       half, fin, s->epi_maps, q);
      else
        nmhd::launch_update(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel, half,
                            fin, q);
    };
    auto whole = [&](int in_sel, int out_sel, int half, int fin) {
      if (s->variant == 3)
        nmhd::launch_cell_stage_chunked(g, s->ctl, s->w0, s->w1, s->wp, s->flux, s->dt_hist, in_sel, out_sel,
                                        half, fin, s->shape.zc, q);
    };
    if (midpoint) {
      flux_k(0, 1);
      whole(0, 2, 1, 0);
      NMHD_CUDA(s, cudaEventRecord(ev[3], q));
      upd_k(0, 2, 1, 0);
      if (s->cfg.flags & NMHD_FLAG_HALO_PER_STAGE) nmhd::launch_fill_predictor(g, s->ctl, s->wp, q);
      NMHD_CUDA(s, cudaEventRecord(ev[4], q));
      flux_k(2, 0);
      whole(2, 1, 0, 1);
      NMHD_CUDA(s, cudaEventRecord(ev[5], q));
      upd_k(2, 1, 0, 1);
    } else {
      NMHD_CUDA(s, cudaEventRecord(ev[3], q));
      NMHD_CUDA(s, cudaEventRecord(ev[4], q));
      flux_k(0, 0);
      whole(0, 1, 0, 1);
      NMHD_CUDA(s, cudaEventRecord(ev[5], q));
      upd_k(0, 1, 0, 1);
    }
    NMHD_CUDA(s, cudaEventRecord(ev[6], q));
    NMHD_CUDA(s, cudaEventSynchronize(ev[6]));
    for (int k = 0; k < kKernelClasses; ++k) {
      float ms = 0.f;
      NMHD_CUDA(s, cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      acc[k] += ms;
    }
    // kernel launches of each class: fill (Y and Z margins), margin CFL, and
    // per stage the flux class (variant 3: the whole chunked stage) and the
    // update class (variant 2: CT + conserved update, variants 4 and 5: the
    // two fused; the per-stage predictor refill is timed with the first
    // stage's update)
    const int fills = (g.my > 0) + (g.mz > 0);
    const int nch = s->variant == 3 ? (g.sz + (s->shape.zc < 1 ? g.sz : s->shape.zc) - 1) /
                                          (s->shape.zc < 1 ? g.sz : s->shape.zc)
                                    : 0;
    const int flux_n = s->variant == 3 ? 3 * nch : 1;
    const int upd_n = s->variant == 3 ? 0 : (s->variant == 2 ? 2 : 1);  // variants 0, 1, 4, 5: one
    cnt[0] += fills;
    cnt[1] += margins;
    cnt[2] += midpoint ? flux_n : 0;
    cnt[3] += midpoint ? upd_n + ((s->cfg.flags & NMHD_FLAG_HALO_PER_STAGE) ? fills : 0) : 0;
    cnt[4] += flux_n;
    cnt[5] += upd_n;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  NMHD_CUDA(s, cudaGetLastError());
  st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  if (h.status) return fail(s, NMHD_ERR_NUMERICAL, "numerical error while profiling");
  const int k = max < kKernelClasses ? max : kKernelClasses;
  for (int i = 0; i < k; ++i) {
    ms_out[i] = acc[i] / steps;
    if (launches_out) launches_out[i] = cnt[i] / steps;
  }
  return k;
}

nmhd_status nmhd_set_kernel(nmhd_solver *s, int variant, int tile_rows, int z_chunk) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  if (variant < 0 || variant > 5) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "variant must be 0 to 5");
  if ((s->cfg.flags & NMHD_FLAG_FAST_ARITHMETIC) && variant != 2 && variant != 4 && variant != 5)
    return fail(s, NMHD_ERR_NOT_SUPPORTED, "fast arithmetic exists for kernel variants 2, 4 and 5 only");
  if (variant == 0 && tile_rows != 4 && tile_rows != 8 && tile_rows != 16)
    return fail(s, NMHD_ERR_INVALID_ARGUMENT, "tile_rows must be 4, 8 or 16");
  if (z_chunk < 0) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "z_chunk must be >= 0");
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  drop_graphs(s);
  s->variant = variant;
  if (variant == 0) s->shape = nmhd::TileShape{tile_rows, z_chunk};
  if (variant == 3) s->shape = nmhd::TileShape{8, z_chunk};
  return NMHD_OK;
}

nmhd_status nmhd_get_kernel(const nmhd_solver *s, int *variant, int *tile_rows, int *z_chunk) {
  if (!s) return NMHD_ERR_INVALID_ARGUMENT;
  if (variant) *variant = s->variant;
  if (tile_rows) *tile_rows = s->shape.ty;
  if (z_chunk) *z_chunk = s->shape.zc;
  return NMHD_OK;
}

}  // extern "C"

namespace {
struct TuneKey {
  int sx, sy, sz, my, mz, problem, so, to;
  bool operator<(const TuneKey &o) const {
    return std::tie(sx, sy, sz, my, mz, problem, so, to) <
           std::tie(o.sx, o.sy, o.sz, o.my, o.mz, o.problem, o.so, o.to);
  }
};
struct TuneChoice {
  int variant, rows, zc;
};
std::map<TuneKey, TuneChoice> g_tune_cache;
std::mutex g_tune_mutex;  // solvers may be created and tuned from several host threads

TuneKey tune_key(const nmhd_solver *s) {
  const GridParams &g = s->g;
  return TuneKey{g.sx, g.sy, g.sz, g.my, g.mz, s->cfg.problem, s->cfg.space_order,
                 s->cfg.time_order + 8 * s->cfg.flags};
}
}  // namespace

void apply_tuned(nmhd_solver *s) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tune_cache.find(tune_key(s));
  if (it == g_tune_cache.end()) return;
  s->variant = it->second.variant;
  s->shape = nmhd::TileShape{it->second.rows, it->second.zc};
}

extern "C" {

int nmhd_autotune(nmhd_solver *s, int steps, double *trials_out, int max_trials) {
  if (!s || steps <= 0) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "bad argument");
  if (s->cfg.parallel_size_y > 1)
    return fail(s, NMHD_ERR_NOT_SUPPORTED, "a radial slab steps through nmhd_halo_pack/unpack and nmhd_step_stages");
  const GridParams &g = s->g;
  const TuneKey key = tune_key(s);
  std::vector<TuneChoice> cands;
  // with fast arithmetic variants 2, 4 and 5 run the fast flux kernel
  // (5 is then 4) and the others do not exist
  const bool fast = (s->cfg.flags & NMHD_FLAG_FAST_ARITHMETIC) != 0;
  if (!fast) cands.push_back({5, 8, 0});
  cands.push_back({4, 8, 0});
  cands.push_back({2, 8, 0});
  if (!fast) {
    cands.push_back({1, 8, 0});
    for (int zc : {4, 8, 16})
      if (zc < g.sz) cands.push_back({3, 8, zc});
    for (int rows : {4, 8, 16})
      for (int zc : {0, 8, 16, 32})
        if (zc == 0 || zc < g.sz) cands.push_back({0, rows, zc});
  }
  // save the state and the clock; every trial starts from them
  StepCtl h0;
  nmhd_status st = read_ctl(s, h0);
  if (st != NMHD_OK) return st;
  const size_t bytes = sizeof(float) * 8 * (size_t)g.n;
  float *saved = nullptr;
  NMHD_CUDA(s, cudaMalloc(&saved, bytes));
  cudaError_t e = cudaMemcpyAsync(saved, current_buffer(s, h0), bytes, cudaMemcpyDeviceToDevice, s->stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int saved_variant = s->variant;
  const nmhd::TileShape saved_shape = s->shape;
  double best = 1e30;
  TuneChoice choice = {saved_variant, saved_shape.ty, saved_shape.zc};
  int written = 0;
  for (size_t c = 0; c < cands.size() && e == cudaSuccess; ++c) {
    s->variant = cands[c].variant;
    s->shape = nmhd::TileShape{cands[c].rows, cands[c].zc};
    StepCtl h = h0;
    h.goal = INFINITY;
    h.done = 0;
    h.status = 0;
    h.blocks_done = 0;
    h.cfl_cur = h.cfl_next = 0x7f800000u;
    e = cudaMemcpyAsync(s->ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(current_buffer(s, h0), saved, bytes, cudaMemcpyDeviceToDevice, s->stream);
    if (e != cudaSuccess) break;
    nmhd::launch_fill(g, s->ctl, s->w0, s->w1, s->stream);
    nmhd::launch_cfl_all(g, s->ctl, s->w0, s->w1, s->stream);
    enqueue_step(s);  // warm-up step
    e = cudaEventRecord(e0, s->stream);
    for (int i = 0; i < steps && e == cudaSuccess; ++i) enqueue_step(s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) break;
    StepCtl hr;
    if (cudaMemcpy(&hr, s->ctl, sizeof(hr), cudaMemcpyDeviceToHost) != cudaSuccess || hr.status) continue;
    const double per = ms / steps;
    if (trials_out && written < max_trials) {
      trials_out[4 * written + 0] = cands[c].variant;
      trials_out[4 * written + 1] = cands[c].rows;
      trials_out[4 * written + 2] = cands[c].zc;
      trials_out[4 * written + 3] = per;
      ++written;
    }
    if (per < best) {
      best = per;
      choice = cands[c];
    }
  }
  // restore the state, the clock and the CFL of the saved state
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->ctl, &h0, sizeof(h0), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(current_buffer(s, h0), saved, bytes, cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(saved);
  if (e != cudaSuccess) {
    s->variant = saved_variant;
    s->shape = saved_shape;
    return cuda_fail(s, e, "nmhd_autotune");
  }
  s->cfl_ready = false;
  drop_graphs(s);
  s->variant = choice.variant;
  s->shape = nmhd::TileShape{choice.rows, choice.zc};
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = choice;
  }
  return written;
}

int nmhd_device(const nmhd_solver *s) { return s ? s->device : -1; }

nmhd_status nmhd_set_stream(nmhd_solver *s, void *cuda_stream) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  NMHD_CUDA(s, cudaStreamSynchronize(s->stream));
  drop_graphs(s);
  if (s->own_stream) cudaStreamDestroy(s->stream);
  s->own_stream = cuda_stream == nullptr;
  if (s->own_stream) {
    NMHD_CUDA(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  } else {
    s->stream = (cudaStream_t)cuda_stream;
  }
  return NMHD_OK;
}

// ---------------------------------------------------------------------------
// Split-phase step of a radial slab (MHDSolver::proceed with kParallelSizeY
// ranks, mhd_solver.inlrb:850-993, communicate() :283-493).

int64_t nmhd_halo_count(const nmhd_solver *s) {
  return s ? (int64_t)8 * s->g.sx * s->g.my * s->g.sz : -1;
}

nmhd_status nmhd_slab_begin(nmhd_solver *s, double goal_time) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  if (h.status) return fail(s, NMHD_ERR_NUMERICAL, "state is not valid (set a new state)");
  h.goal = (float)goal_time;
  h.done = 0;
  if (!s->cfl_ready) {
    h.cfl_cur = h.cfl_next = 0x7f800000u;
    h.blocks_done = 0;
  }
  return write_ctl(s, h);
}

nmhd_status nmhd_halo_pack(nmhd_solver *s, float *send_inc, float *send_dec) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  if (s->g.my > 0 && (!send_inc || !send_dec)) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL halo buffer");
  nmhd::launch_halo_pack(s->g, s->ctl, s->w0, s->w1, send_inc, send_dec, s->stream);
  NMHD_CUDA(s, cudaGetLastError());
  return NMHD_OK;
}

nmhd_status nmhd_halo_unpack(nmhd_solver *s, const float *recv_inc, const float *recv_dec) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  if (s->g.my > 0 && (!recv_inc || !recv_dec)) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL halo buffer");
  nmhd::launch_halo_unpack(s->g, s->ctl, s->w0, s->w1, recv_inc, recv_dec, s->stream);
  // the CFL time of this slab: every cell after a state change, else the
  // margin set (the interior was reduced by the previous step's final stage)
  if (!s->cfl_ready) {
    nmhd::launch_cfl_all(s->g, s->ctl, s->w0, s->w1, s->stream);
    s->cfl_ready = true;
  } else {
    nmhd::launch_cfl_margin(s->g, s->ctl, s->w0, s->w1, s->stream);
  }
  NMHD_CUDA(s, cudaGetLastError());
  return NMHD_OK;
}

float *nmhd_cfl_slot(nmhd_solver *s) { return s ? reinterpret_cast<float *>(&s->ctl->cfl_cur) : nullptr; }

nmhd_status nmhd_cfl_min(nmhd_solver *const *slabs, int n) {
  if (!slabs || n < 1 || n > nmhd::kMaxSlots) return fail(nullptr, NMHD_ERR_INVALID_ARGUMENT, "bad slab list");
  nmhd::CflSlots slots;
  slots.n = n;
  for (int i = 0; i < n; ++i) {
    if (!slabs[i] || slabs[i]->device != slabs[0]->device || slabs[i]->stream != slabs[0]->stream)
      return fail(slabs[0], NMHD_ERR_INVALID_ARGUMENT, "slabs must share one device and one stream");
    slots.p[i] = nmhd_cfl_slot(slabs[i]);
  }
  nmhd::launch_cfl_min(slots, slabs[0]->stream);
  NMHD_CUDA(slabs[0], cudaGetLastError());
  return NMHD_OK;
}

nmhd_status nmhd_step_stages(nmhd_solver *s) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  if (s->cfg.time_order == 1) {
    enqueue_stage(s, 0, 1, 0, 1, s->stream);
  } else {
    enqueue_stage(s, 0, 2, 1, 0, s->stream);
    if (s->cfg.flags & NMHD_FLAG_HALO_PER_STAGE) nmhd::launch_fill_predictor(s->g, s->ctl, s->wp, s->stream);
    enqueue_stage(s, 2, 1, 0, 1, s->stream);
  }
  NMHD_CUDA(s, cudaGetLastError());
  return NMHD_OK;
}

nmhd_status nmhd_slab_poll(nmhd_solver *s, int64_t *generation, double *time) {
  if (!s) return fail(s, NMHD_ERR_INVALID_ARGUMENT, "NULL solver");
  StepCtl h;
  nmhd_status st = read_ctl(s, h);
  if (st != NMHD_OK) return st;
  if (generation) *generation = h.generation;
  if (time) *time = h.time;
  if (h.status)
    return fail(s, NMHD_ERR_NUMERICAL,
                (h.status & nmhd::kStatusTimeout) ? "a kernel's bounded wait for its tensor copies gave up"
                : (h.status & nmhd::kStatusBadDt) ? "time step is negative or not finite"
                                                  : "non-finite state, density <= 0 or pressure <= 0");
  return h.done ? NMHD_GOAL_REACHED : NMHD_OK;
}

const char *nmhd_last_error(const nmhd_solver *s) {
  return s ? s->err.c_str() : g_create_error.c_str();
}

}  // extern "C"
