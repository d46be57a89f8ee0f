// Host build of the differentiated step, for the CPU tests only.
//
// Runs the same functors and step drivers as the CUDA adjoint kernels
// (nmhd_b200/csrc/ad_driver.cuh) with a host executor that loops over the
// cells, so the tests can check on a CPU that
//  - the generic forward reproduces the oracle (float and double, bitwise),
//  - the tangent-linear step matches central differences,
//  - the hand-written adjoint is the exact transpose of the tangent-linear
//    step (dot-product test),
// on small boxes.  Not part of the library; nothing in nmhd_b200 loads it.
#include <cstring>
#include <vector>

#include "../../nmhd_b200/csrc/ad_driver.cuh"

using namespace nmhd::ad;

namespace {

struct HostExec {
  template <class R, class F>
  void cells(const GGrid<R> &g, const F &f) {
    for (int z = 0; z < g.sz; ++z)
      for (int y = 0; y < g.sy; ++y)
        for (int x = 0; x < g.sx; ++x) f(x, y, z);
  }
  template <class F>
  void items(int n, const F &f) {
    for (int i = 0; i < n; ++i) f(i);
  }
  template <class T>
  void zero(T *p, size_t n) {
    for (size_t i = 0; i < n; ++i) p[i] = T();
  }
};

template <class T, class R>
typename Wide64<T>::type stress(const GGrid<R> &g, const T *w) {
  typedef typename Wide64<T>::type D;
  D acc = to<D>(0.0);
  for (int z = 0; z < g.sz; ++z)
    for (int y = 0; y < g.sy; ++y)
      for (int x = 0; x < g.sx; ++x) acc = acc + g_stress_cell(g, w, x, y, z);
  return acc;
}

HState<double> unpack(const double in[14]) {
  HState<double> s;
  s.dl = in[0]; s.dr = in[1]; s.ul = in[2]; s.ur = in[3]; s.vl = in[4]; s.vr = in[5]; s.wl = in[6];
  s.wr = in[7]; s.pl = in[8]; s.pr = in[9]; s.byl = in[10]; s.byr = in[11]; s.bzl = in[12]; s.bzr = in[13];
  return s;
}
template <class R>
void pack(const HState<R> &s, R out[14]) {
  const R v[14] = {s.dl, s.dr, s.ul, s.ur, s.vl, s.vr, s.wl, s.wr, s.pl, s.pr, s.byl, s.byr, s.bzl, s.bzr};
  for (int i = 0; i < 14; ++i) out[i] = v[i];
}
template <class R>
HState<R> unpack_r(const R in[14]) {
  HState<R> s;
  R *p = &s.dl;
  for (int i = 0; i < 14; ++i) p[i] = in[i];
  return s;
}

// Forward over nsteps steps with frozen dt (T = float or double).
template <class T>
void forward(const nmhd_config &c, T *state, double time, const T *dts, int nsteps) {
  HostExec ex;
  const GGrid<T> g = make_ggrid<T>(c);
  const size_t n = (size_t)g.n;
  std::vector<T> tape((size_t)kTapeFields * n), fscr((size_t)kFluxScratchFields * n);
  StepTape<T> t = tape_at(tape.data(), n, fscr.data());
  std::memcpy(t.wf, state, sizeof(T) * 8 * n);
  for (int i = 0; i < nsteps; ++i) {
    fwd_step(ex, g, c.time_order, time, dts[i], t);
    time = time + (double)dts[i];
    std::memcpy(t.wf, t.wo, sizeof(T) * 8 * n);
  }
  std::memcpy(state, t.wf, sizeof(T) * 8 * n);
}

}  // namespace

extern "C" {

void adh_hlld_f32(float gamma, float bx, const float in[14], float out[7]) {
  hlld_g(gamma, bx, unpack_r(in), out);
}
void adh_hlld_f64(double gamma, double bx, const double in[14], double out[7]) {
  hlld_g(gamma, bx, unpack(in), out);
}
// Tangent of the HLLD flux along (din, dbx).
void adh_hlld_tan(double gamma, double bx, const double in[14], double dbx, const double din[14], double out[7],
                  double dout[7]) {
  typedef Dual<double> D;
  HState<D> s;
  D *p = &s.dl;
  for (int i = 0; i < 14; ++i) p[i] = D(in[i], din[i]);
  D f[7];
  hlld_g(D(gamma), D(bx, dbx), s, f);
  for (int i = 0; i < 7; ++i) {
    out[i] = f[i].v;
    dout[i] = f[i].d;
  }
}
void adh_hlld_adj_f64(double gamma, double bx, const double in[14], const double lf[7], double lin[14],
                      double *lbx) {
  HState<double> ls;
  hlld_adjoint(gamma, bx, unpack(in), lf, ls, *lbx);
  pack(ls, lin);
}
void adh_hlld_adj_f32(float gamma, float bx, const float in[14], const float lf[7], float lin[14], float *lbx) {
  HState<float> ls;
  hlld_adjoint(gamma, bx, unpack_r(in), lf, ls, *lbx);
  pack(ls, lin);
}
int adh_hlld_region_f32(float gamma, float bx, const float in[14]) {
  HTape<float> t;
  hlld_tape(gamma, bx, unpack_r(in), t);
  return t.region;
}

void adh_forward_f32(const nmhd_config *c, float *state, double time, const float *dts, int nsteps) {
  forward<float>(*c, state, time, dts, nsteps);
}
void adh_forward_f64(const nmhd_config *c, double *state, double time, const double *dts, int nsteps) {
  forward<double>(*c, state, time, dts, nsteps);
}

// FP64 tangent-linear run: J and dJ[dir] (dir may be NULL).
void adh_tlm(const nmhd_config *c, const double *state, const double *dir, double time, const double *dts,
             int nsteps, const nmhd_loss_spec *l, double *loss, double *dloss) {
  typedef Dual<double> D;
  HostExec ex;
  const GGrid<double> g = make_ggrid<double>(*c);
  const size_t n = (size_t)g.n;
  std::vector<D> tape((size_t)kTapeFields * n), fscr((size_t)kFluxScratchFields * n);
  StepTape<D> t = tape_at(tape.data(), n, fscr.data());
  for (size_t i = 0; i < 8 * n; ++i) t.wf[i] = D(state[i], dir ? dir[i] : 0.0);
  D acc(0.0);
  if (in_window(*l, 0)) acc = acc + stress(g, t.wf);
  for (int i = 0; i < nsteps; ++i) {
    fwd_step(ex, g, c->time_order, time, dts[i], t);
    time = time + dts[i];
    if (in_window(*l, i + 1)) acc = acc + stress(g, t.wo);
    std::memcpy(t.wf, t.wo, sizeof(D) * 8 * n);
  }
  const double s = stress_scale(*c, *l);
  *loss = acc.v * s;
  *dloss = acc.d * s;
}

}  // extern "C"

// Adjoint run (R = float or double) storing every step's tape.
template <class R>
static void adjoint(const nmhd_config &c, const R *state, double time, const R *dts, int nsteps,
                    const nmhd_loss_spec &l, double *loss, R *grad) {
  HostExec ex;
  const GGrid<R> g = make_ggrid<R>(c);
  const size_t n = (size_t)g.n;
  std::vector<R> tapes((size_t)nsteps * kTapeFields * n), fscr((size_t)kFluxScratchFields * n);
  std::vector<double> tn(nsteps + 1);
  tn[0] = time;
  double acc = 0.0;
  std::memcpy(tapes.data(), state, sizeof(R) * 8 * n);
  if (in_window(l, 0)) acc += stress(g, state);
  for (int i = 0; i < nsteps; ++i) {
    StepTape<R> t = tape_at(tapes.data() + (size_t)i * kTapeFields * n, n, fscr.data());
    fwd_step(ex, g, c.time_order, tn[i], dts[i], t);
    tn[i + 1] = tn[i] + (double)dts[i];
    if (in_window(l, i + 1)) acc += stress(g, t.wo);
    if (i + 1 < nsteps) std::memcpy(tapes.data() + (size_t)(i + 1) * kTapeFields * n, t.wo, sizeof(R) * 8 * n);
  }
  const double s = stress_scale(c, l);
  *loss = acc * s;
  std::vector<R> lam(24 * n), scr((size_t)kAdjScratchFields * n);
  R *lamA = lam.data(), *lamS = lamA + 8 * n, *lamF = lamA + 16 * n;
  const AdjScratch<R> sc = scratch_at(scr.data(), n);
  ex.zero(lamA, 8 * n);
  for (int i = nsteps - 1; i >= 0; --i) {
    StepTape<R> t = tape_at(tapes.data() + (size_t)i * kTapeFields * n, n, fscr.data());
    if (in_window(l, i + 1)) ex.cells(g, OpAStress<R>{g, t.wo, lamA, s});
    adj_step(ex, g, c.time_order, tn[i], dts[i], t, lamA, lamS, lamF, sc);
    R *tmp = lamA;
    lamA = lamF;
    lamF = tmp;
  }
  if (in_window(l, 0)) ex.cells(g, OpAStress<R>{g, state, lamA, s});
  std::memcpy(grad, lamA, sizeof(R) * 8 * n);
}

extern "C" {

void adh_adjoint_f64(const nmhd_config *c, const double *state, double time, const double *dts, int nsteps,
                     const nmhd_loss_spec *l, double *loss, double *grad) {
  adjoint<double>(*c, state, time, dts, nsteps, *l, loss, grad);
}
void adh_adjoint_f32(const nmhd_config *c, const float *state, double time, const float *dts, int nsteps,
                     const nmhd_loss_spec *l, double *loss, float *grad) {
  adjoint<float>(*c, state, time, dts, nsteps, *l, loss, grad);
}

}  // extern "C"
