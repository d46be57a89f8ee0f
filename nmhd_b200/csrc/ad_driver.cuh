// Step-level drivers of the differentiated time step, written once over an
// executor: the CUDA executor (adjoint.cu) launches one kernel per pass; the
// host executor of the tests' check harness loops over the same functors.
//
//   fwd_step   one RK2 (or Euler) step with a frozen dt over scalar T
//              (double: FP64 step, Dual<double>: tangent-linear step), keeping
//              the filled input, the predictor, the raw output and both stages'
//              face fluxes - the tape the adjoint reads;
//   adj_step   the transpose of that step: adjoint of the raw output -> adjoint
//              of the step's input, through both stages and the margin fill.
#pragma once
#include <cstddef>

#include "../../include/nmhd.h"
#include "ad_cell.cuh"

namespace nmhd {
namespace ad {

// Number of fields of one step's tape: filled input (8), predictor (8), raw
// output (8).  The stages' face fluxes go to one shared scratch of 21 fields:
// the adjoint recomputes what it needs of them.
constexpr int kTapeFields = 24;
constexpr int kFluxScratchFields = 21;
// Scratch fields of the adjoint of a stage: lamU 5, lamE 1, lamBn 3, face 30, lamBc 3.
constexpr int kAdjScratchFields = 42;

template <class T>
struct StepTape {
  T *wf, *f1, *ws, *f2, *wo;
};

template <class T>
StepTape<T> tape_at(T *base, size_t n, T *flux_scratch) {
  StepTape<T> t;
  t.wf = base;
  t.ws = base + 8 * n;
  t.wo = base + 16 * n;
  t.f1 = t.f2 = flux_scratch;
  return t;
}

template <class R>
struct AdjScratch {
  R *lamU, *lamE, *lamBn, *face, *lamBc;
};

template <class R>
AdjScratch<R> scratch_at(R *base, size_t n) {
  AdjScratch<R> s;
  s.lamU = base;
  s.lamE = base + 5 * n;
  s.lamBn = base + 6 * n;
  s.face = base + 9 * n;
  s.lamBc = base + 39 * n;
  return s;
}

// The reference's derived constants evaluated in precision R
// (simulation_config_default.h:56-103; relative_velocity of
// src/application/kepler_disk_demo/mhd_solver.curb:50-52).
template <class R>
GGrid<R> make_ggrid(const nmhd_config &c) {
  GGrid<R> g;
  g.sx = c.size_x;
  g.sy = c.size_y;
  g.sz = c.size_z;
  g.n = c.size_x * c.size_y * c.size_z;
  g.my = c.margin_y;
  g.mz = c.margin_z;
  g.shear = c.problem == NMHD_PROBLEM_SHEARING_BOX;
  g.order2 = c.space_order != 1;
  const int s[3] = {c.size_x, c.size_y, c.size_z};
  const int gi[3] = {c.size_x, c.size_y - 2 * c.margin_y, c.size_z - 2 * c.margin_z};
  const float L[3] = {c.extent_x, c.extent_y, c.extent_z};
  volatile R comp[3], local[3], d[3];
  for (int i = 0; i < 3; ++i) {
    volatile R per = (R)L[i] / (R)gi[i];
    comp[i] = per * (R)s[i];
    local[i] = per * (R)gi[i];
    d[i] = comp[i] / (R)s[i];
  }
  g.dx = d[0];
  g.dy = d[1];
  g.dz = d[2];
  g.idx = (R)1 / g.dx;
  g.idy = (R)1 / g.dy;
  g.idz = (R)1 / g.dz;
  g.extent_x = comp[0];
  g.corner_y = -comp[1] / (R)2;
  g.gamma = (R)c.gamma;
  g.cfl = (R)c.cfl;
  g.q = (R)c.q;
  g.omega = (R)c.omega;
  volatile R qo = -g.q * g.omega;
  volatile R rv = qo * local[1];
  g.rel_vel = (double)rv;
  return g;
}

// ---------------------------------------------------------------------------
// Functors (one pass each)
template <class T, class R>
struct OpFillY {
  GGrid<R> g;
  double time;
  T *w;
  NMHD_HD void operator()(int i) const { g_fill_y_item(g, time, w, i); }
};
template <class T, class R>
struct OpFillZ {
  GGrid<R> g;
  T *w;
  NMHD_HD void operator()(int i) const { g_fill_z_item(g, w, i); }
};
template <class T, class R>
struct OpFlux {
  GGrid<R> g;
  const T *w;
  T *flux;
  T h;
  NMHD_HD void operator()(int x, int y, int z) const { g_flux_cell(g, w, flux, x, y, z, h); }
};
template <class T, class R>
struct OpCt {
  GGrid<R> g;
  const T *win, *wb;
  T *wo;
  const T *flux;
  T h;
  NMHD_HD void operator()(int x, int y, int z) const { g_ct_cell(g, win, wb, wo, flux, x, y, z, h); }
};
template <class T, class R>
struct OpPrim {
  GGrid<R> g;
  const T *wb;
  T *wo;
  const T *flux;
  T h;
  NMHD_HD void operator()(int x, int y, int z) const { g_prim_cell(g, wb, wo, flux, x, y, z, h); }
};
template <class T, class R>
struct OpStress {
  GGrid<R> g;
  const T *w;
  NMHD_HD typename Wide64<T>::type operator()(int x, int y, int z) const { return g_stress_cell(g, w, x, y, z); }
};

template <class R>
struct OpAPrim {
  GGrid<R> g;
  const R *wb, *wo, *lout;
  R *lamU, *lamE, *lb;
  R h;
  NMHD_HD void operator()(int x, int y, int z) const { a_prim_cell(g, wb, wo, lout, lamU, lamE, lb, x, y, z, h); }
};
template <class R>
struct OpABface {
  GGrid<R> g;
  const R *wb, *wo, *lout, *lamU, *lamE;
  R *lamBn, *lb;
  R *lamBc;  // cleared here for the reconstruction passes that follow
  NMHD_HD void operator()(int x, int y, int z) const {
    a_bface_cell(g, wb, wo, lout, lamU, lamE, lamBn, lb, x, y, z);
    const size_t N = (size_t)g.n;
    const int o = cell_at(g, x, y, z);
    lamBc[o] = R(0);
    lamBc[N + o] = R(0);
    lamBc[2 * N + o] = R(0);
  }
};
template <class R, int AX>
struct OpAFlux {
  GGrid<R> g;
  const R *win, *lamBn, *lamU;
  R *face;
  R h;
  NMHD_HD void operator()(int x, int y, int z) const { a_flux_face<AX>(g, win, lamBn, lamU, face, x, y, z, h); }
};
template <class R, int AX>
struct OpARecon {
  GGrid<R> g;
  const R *face;
  R *lin, *lamBc;
  R h;
  NMHD_HD void operator()(int x, int y, int z) const { a_recon_face<AX>(g, face, lin, lamBc, x, y, z, h); }
};
template <class R>
struct OpABc {
  GGrid<R> g;
  const R *lamBc;
  R *lin;
  NMHD_HD void operator()(int x, int y, int z) const { a_bc_cell(g, lamBc, lin, x, y, z); }
};
template <class R>
struct OpAFillY {
  GGrid<R> g;
  int dint;
  R f;
  R *lam;
  NMHD_HD void operator()(int i) const { a_fill_y_item(g, dint, f, lam, i); }
};
template <class R>
struct OpAFillZ {
  GGrid<R> g;
  R *lam;
  NMHD_HD void operator()(int i) const { a_fill_z_item(g, lam, i); }
};
template <class R>
struct OpAStress {
  GGrid<R> g;
  const R *w;
  R *lam;
  double s;
  NMHD_HD void operator()(int x, int y, int z) const { a_stress_cell(g, w, lam, x, y, z, s); }
};

// ---------------------------------------------------------------------------
// Forward
template <class Ex, class T, class R>
void fwd_fill(Ex &ex, const GGrid<R> &g, double time, T *w) {
  if (g.my > 0) ex.items(g.sx * g.my * g.sz, OpFillY<T, R>{g, time, w});
  if (g.mz > 0) ex.items(g.sx * g.sy * g.mz, OpFillZ<T, R>{g, w});
}

template <class Ex, class T, class R>
void fwd_stage(Ex &ex, const GGrid<R> &g, const T *win, const T *wb, T *wo, T *flux, const T &h) {
  ex.cells(g, OpFlux<T, R>{g, win, flux, h});
  ex.cells(g, OpCt<T, R>{g, win, wb, wo, flux, h});
  ex.cells(g, OpPrim<T, R>{g, wb, wo, flux, h});
}

// One step: t.wf holds W^n on entry (its margins are filled in place); the
// raw W^{n+1} goes to t.wo.
template <class Ex, class T, class R>
void fwd_step(Ex &ex, const GGrid<R> &g, int time_order, double time, R dt, const StepTape<T> &t) {
  fwd_fill(ex, g, time, t.wf);
  if (time_order == 1) {
    fwd_stage(ex, g, t.wf, t.wf, t.wo, t.f1, to<T>(dt));
  } else {
    fwd_stage(ex, g, t.wf, t.wf, t.ws, t.f1, to<T>(dt / R(2)));
    fwd_stage(ex, g, t.ws, t.wf, t.wo, t.f2, to<T>(dt));
  }
}

// ---------------------------------------------------------------------------
// Adjoint
template <class Ex, class R>
void adj_stage(Ex &ex, const GGrid<R> &g, const R *win, const R *wb, const R *wo, R h, const R *lout, R *lin,
               R *lb, const AdjScratch<R> &sc) {
  ex.cells(g, OpAPrim<R>{g, wb, wo, lout, sc.lamU, sc.lamE, lb, h});
  ex.cells(g, OpABface<R>{g, wb, wo, lout, sc.lamU, sc.lamE, sc.lamBn, lb, sc.lamBc});
  // one face axis at a time through the shared face scratch
  ex.cells(g, OpAFlux<R, 0>{g, win, sc.lamBn, sc.lamU, sc.face, h});
  ex.cells(g, OpARecon<R, 0>{g, sc.face, lin, sc.lamBc, h});
  ex.cells(g, OpAFlux<R, 1>{g, win, sc.lamBn, sc.lamU, sc.face, h});
  ex.cells(g, OpARecon<R, 1>{g, sc.face, lin, sc.lamBc, h});
  ex.cells(g, OpAFlux<R, 2>{g, win, sc.lamBn, sc.lamU, sc.face, h});
  ex.cells(g, OpARecon<R, 2>{g, sc.face, lin, sc.lamBc, h});
  ex.cells(g, OpABc<R>{g, sc.lamBc, lin});
}

// Adjoint of one step recorded in tape t: lam_next is the adjoint of t.wo
// (read only); on return lam_f holds the adjoint of the step's input W^n.
// lam_s is scratch (the predictor's adjoint).
template <class Ex, class R>
void adj_step(Ex &ex, const GGrid<R> &g, int time_order, double time, R dt, const StepTape<R> &t,
              const R *lam_next, R *lam_s, R *lam_f, const AdjScratch<R> &sc) {
  const size_t n8 = (size_t)8 * g.n;
  ex.zero(lam_f, n8);
  if (time_order == 1) {
    adj_stage(ex, g, t.wf, t.wf, t.wo, dt, lam_next, lam_f, lam_f, sc);
  } else {
    ex.zero(lam_s, n8);
    adj_stage(ex, g, t.ws, t.wf, t.wo, dt, lam_next, lam_s, lam_f, sc);
    adj_stage(ex, g, t.wf, t.wf, t.ws, dt / R(2), lam_s, lam_f, lam_f, sc);
  }
  // margin fill: W_f = Fz(Fy(W^n)), so apply Fz^T then Fy^T
  if (g.mz > 0) ex.items(g.sx * g.sy * g.mz, OpAFillZ<R>{g, lam_f});
  if (g.my > 0) {
    int dint;
    R f;
    shear_shift(g, time, dint, f);
    ex.items(g.sx * g.my * g.sz, OpAFillY<R>{g, dint, f, lam_f});
  }
}

// Loss: J = s * sum over the window's states of sum_cells -(Bx By)_centre,
// s = 1 / (interior cells * window length).
inline double stress_scale(const nmhd_config &c, const nmhd_loss_spec &l) {
  const double cells = (double)c.size_x * (c.size_y - 2 * c.margin_y) * (c.size_z - 2 * c.margin_z);
  return 1.0 / (cells * (double)(l.last_step - l.first_step + 1));
}

inline bool in_window(const nmhd_loss_spec &l, int n) { return n >= l.first_step && n <= l.last_step; }

}  // namespace ad
}  // namespace nmhd
