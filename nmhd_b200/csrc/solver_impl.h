// Host-side state of one nmhd_solver handle, shared by the translation units
// that implement its C ABI (solver.cu: stepping, I/O, autotuning; adjoint.cu:
// differentiation).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>

#include "../../include/nmhd.h"
#include "step.cuh"

struct nmhd_solver {
  nmhd_config cfg;
  nmhd::GridParams g;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  float *w0 = nullptr, *w1 = nullptr, *wp = nullptr, *flux = nullptr, *dt_hist = nullptr;
  nmhd::StepCtl *ctl = nullptr;
  double *diag = nullptr;
  bool cfl_ready = false;  // ctl->cfl_cur holds the CFL time of the current state
  // 0: z-marching tiled kernels, 1: per-cell 1-D, 2: per-cell 3-D blocks,
  // 3: variant 2 as a z-chunk pipeline, 4: the variant-2 flux kernel with the
  // fused stage epilogue, 5 (the default): the staged flux kernel with the
  // fused stage epilogue
  int variant = 5;
  nmhd::TileShape shape = {8, 16};
  std::map<int, cudaGraphExec_t> graphs;
  // Pinned copies of the control block after each of the (at most two) step
  // batches in flight in nmhd_proceed, and the events that mark them.
  nmhd::StepCtl *hctl = nullptr;
  cudaEvent_t batch_done[2] = {nullptr, nullptr};
  std::string err;
  void *adjoint = nullptr;  // differentiation workspace (adjoint.cu), allocated on first use
  // tensor maps of the fused epilogue and the staged flux kernel (variants
  // 4 and 5) over w0, w1, wp and flux
  nmhd::EpilogueMaps *epi_maps = nullptr;
};

// Frees the differentiation workspace of a handle (adjoint.cu).
void nmhd_adjoint_release(nmhd_solver *s);
