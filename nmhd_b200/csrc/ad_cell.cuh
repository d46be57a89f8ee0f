// Per-cell operations of the differentiated time step.
//
// Forward (generic scalar T, see ad_scalar.cuh): the margin fill and the three
// parts of an RK stage exactly as the production kernels (cell_ops.cuh,
// margin_ops.cuh) evaluate them, operation for operation, with plain
// divisions by the spacing.  With T = float they reproduce the FP32 step,
// with T = double the reference's Real = double build, with T = Dual<double>
// the FP64 tangent-linear step.
//
// Adjoint (real R = float or double): the transpose of the linearised stage
// with dt, the limiter choices, the Riemann fan region and the CT upwind
// choices frozen at the values the forward took.  Every adjoint part is a
// gather (each cell writes only its own entries), so no atomics are needed
// and results are deterministic:
//   a_prim_cell    to_primitive + kick + conserved update (per cell)
//   a_bface_cell   face-B adjoint: output B, energy terms of old and new B
//   a_flux_face    CT transpose and flux divergence transpose -> adjoint of the
//                  7 fluxes of one face of the cell -> HLLD adjoint (per axis)
//   a_recon_face   minbee reconstruction, face kick and normal-B transposes
//                  (per axis)
//   a_bc_cell      transverse cell-centred B average transpose
//   a_fill_*       transpose of the shearing-periodic and Z margin fills
// References: src/library/mhd_solver.inlrb:140-155 (reconstruction), 184-259
// (shear fill), 562-714 (flux, CT), 762-848 (conversions, update, kick).
#pragma once
#include "ad_hlld.cuh"

namespace nmhd {
namespace ad {

// Grid constants in precision R (the reference's derived constants,
// simulation_config_default.h:56-103, evaluated in R).
template <class R>
struct GGrid {
  int sx, sy, sz, n, my, mz, shear, order2;
  R dx, dy, dz, gamma, cfl, q, omega, corner_y, extent_x;
  R idx, idy, idz;  // 1/dx, 1/dy, 1/dz (adjoint only; the forward divides)
  double rel_vel;
};

NMHD_HD int wrapc(int v, int s) {
  while (v < 0) v += s;
  while (v >= s) v -= s;
  return v;
}

template <class R>
NMHD_HD int cell_at(const GGrid<R> &g, int x, int y, int z) {
  return (wrapc(z, g.sz) * g.sy + wrapc(y, g.sy)) * g.sx + wrapc(x, g.sx);
}

// (x, y, z) + k along axis a
template <class R>
NMHD_HD int shifted(const GGrid<R> &g, int x, int y, int z, int a, int k) {
  return cell_at(g, x + (a == 0 ? k : 0), y + (a == 1 ? k : 0), z + (a == 2 ? k : 0));
}

template <class R>
NMHD_HD R spacing(const GGrid<R> &g, int a) {
  return a == 0 ? g.dx : (a == 1 ? g.dy : g.dz);
}

template <class R>
NMHD_HD R inv_spacing(const GGrid<R> &g, int a) {
  return a == 0 ? g.idx : (a == 1 ? g.idy : g.idz);
}

// ---------------------------------------------------------------------------
// Forward
template <class T>
NMHD_HD T absolute_smaller_g(const T &a, const T &b) {
  typedef typename Traits<T>::real R;
  return val(a) * val(b) <= R(0) ? to<T>(R(0)) : (gabs(a) < gabs(b) ? a : b);
}

template <class T>
NMHD_HD void reconstruct4_g(const T &x0, const T &x1, const T &x2, const T &x3, T &left, T &right) {
  const T d01 = x1 - x0;
  const T d12 = x2 - x1;
  const T d23 = x3 - x2;
  const T d1 = absolute_smaller_g(d01, d12);
  const T d2 = absolute_smaller_g(d12, d23);
  left = x1 + d1 / to<T>(2.0f);
  right = x2 - d2 / to<T>(2.0f);
}

// Riemann input of the lower ax-face of cell (x, y, z): reconstruction,
// transverse B averages and the face half-kick (calc_flux_kernel).
template <class T, class R>
NMHD_HD void face_input(const GGrid<R> &g, const T *w, int x, int y, int z, int ax, const T &h, HState<T> &in,
                        T &bn) {
  const size_t N = (size_t)g.n;
  const int e1 = ax == 2 ? 0 : ax + 1, e2 = ax == 0 ? 2 : ax - 1;
  int c[4];
  for (int t = 0; t < 4; ++t) c[t] = shifted(g, x, y, z, ax, t - 2);
  const T *rho = w, *p = w + 4 * N;
  const T *vn = w + (1 + ax) * N, *v1 = w + (1 + e1) * N, *v2 = w + (1 + e2) * N;
  const T *b1 = w + (5 + e1) * N, *b2 = w + (5 + e2) * N;
  T bc1[4], bc2[4];
  for (int t = 0; t < 4; ++t) {
    const int cx = x + (ax == 0 ? t - 2 : 0), cy = y + (ax == 1 ? t - 2 : 0), cz = z + (ax == 2 ? t - 2 : 0);
    bc1[t] = to<T>(0.5f) * (b1[c[t]] + b1[shifted(g, cx, cy, cz, e1, 1)]);
    bc2[t] = to<T>(0.5f) * (b2[c[t]] + b2[shifted(g, cx, cy, cz, e2, 1)]);
  }
  if (g.order2) {
    reconstruct4_g(rho[c[0]], rho[c[1]], rho[c[2]], rho[c[3]], in.dl, in.dr);
    reconstruct4_g(vn[c[0]], vn[c[1]], vn[c[2]], vn[c[3]], in.ul, in.ur);
    reconstruct4_g(v1[c[0]], v1[c[1]], v1[c[2]], v1[c[3]], in.vl, in.vr);
    reconstruct4_g(v2[c[0]], v2[c[1]], v2[c[2]], v2[c[3]], in.wl, in.wr);
    reconstruct4_g(p[c[0]], p[c[1]], p[c[2]], p[c[3]], in.pl, in.pr);
    reconstruct4_g(bc1[0], bc1[1], bc1[2], bc1[3], in.byl, in.byr);
    reconstruct4_g(bc2[0], bc2[1], bc2[2], bc2[3], in.bzl, in.bzr);
  } else {
    in.dl = rho[c[1]]; in.dr = rho[c[2]];
    in.ul = vn[c[1]]; in.ur = vn[c[2]];
    in.vl = v1[c[1]]; in.vr = v1[c[2]];
    in.wl = v2[c[1]]; in.wr = v2[c[2]];
    in.pl = p[c[1]]; in.pr = p[c[2]];
    in.byl = bc1[1]; in.byr = bc1[2];
    in.bzl = bc2[1]; in.bzr = bc2[2];
  }
  if (g.shear) {
    T acc;
    if (ax == 0) {
      const T vY = to<T>(0.5f) * (w[2 * N + c[1]] + w[2 * N + c[2]]);
      acc = to<T>(-2.0f) * to<T>(g.omega) * vY;
    } else if (ax == 1) {
      const T vX = to<T>(0.5f) * (w[N + c[1]] + w[N + c[2]]);
      acc = to<T>(2.0f) * to<T>(g.omega) * vX +
            to<T>(R(2.0f) * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((R)y + R(0.5f))));
    } else {
      acc = to<T>(R(0));
    }
    const T mbv = to<T>(0.5f) * h * acc;
    in.ul = in.ul + mbv;
    in.ur = in.ur + mbv;
  }
  bn = w[(5 + ax) * N + c[2]];
}

// The three lower-face fluxes of a cell (7 per face; momentum in absolute
// components, then F(B_e1), F(B_e2)) into flux + (7*ax + k)*N.
template <class T, class R>
NMHD_HD void g_flux_cell(const GGrid<R> &g, const T *w, T *flux, int x, int y, int z, const T &h) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  for (int ax = 0; ax < 3; ++ax) {
    const int e1 = ax == 2 ? 0 : ax + 1, e2 = ax == 0 ? 2 : ax - 1;
    HState<T> in;
    T bn;
    face_input(g, w, x, y, z, ax, h, in, bn);
    T f[7];
    hlld_g(to<T>(g.gamma), bn, in, f);
    T *out = flux + (size_t)(7 * ax) * N + o;
    out[0] = f[0];
    out[(1 + ax) * N] = f[1];
    out[(1 + e1) * N] = f[2];
    out[(1 + e2) * N] = f[3];
    out[4 * N] = f[4];
    out[5 * N] = f[5];
    out[6 * N] = f[6];
  }
}

// Upwind edge flux (corner_magnet_flux): the a-flux of B_b at edge e,
// F[e - b] if the 4-cell wind sum is positive, F[e] if negative, else the mean.
template <class T, class R>
NMHD_HD T g_corner(const GGrid<R> &g, const T *vb, const T *fb, int x, int y, int z, int a, int b) {
  const int e = cell_at(g, x, y, z);
  const int eb = shifted(g, x, y, z, b, -1);
  const int ea = shifted(g, x, y, z, a, -1);
  const int eab = cell_at(g, x - (a == 0 || b == 0), y - (a == 1 || b == 1), z - (a == 2 || b == 2));
  const T w = vb[e] + vb[eb] + vb[ea] + vb[eab];
  typedef typename Traits<T>::real RR;
  const T f0 = fb[eb], f1 = fb[e];
  return val(w) > RR(0) ? f0 : (val(w) < RR(0) ? f1 : to<T>(0.5f) * (f0 + f1));
}

// Face-B update of the cell's three lower faces (constrained transport).
template <class T, class R>
NMHD_HD void g_ct_cell(const GGrid<R> &g, const T *win, const T *wb, T *wo, const T *flux, int x, int y, int z,
                       const T &h) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  const T *vx = win + N, *vy = win + 2 * N, *vz = win + 3 * N;
  const T *FxBy = flux + 5 * N, *FxBz = flux + 6 * N;
  const T *FyBz = flux + 12 * N, *FyBx = flux + 13 * N;
  const T *FzBx = flux + 19 * N, *FzBy = flux + 20 * N;
  const T XY00 = g_corner(g, vy, FxBy, x, y, z, 0, 1), XY01 = g_corner(g, vy, FxBy, x, y + 1, z, 0, 1);
  const T XY10 = g_corner(g, vy, FxBy, x + 1, y, z, 0, 1);
  const T YX00 = g_corner(g, vx, FyBx, x, y, z, 1, 0), YX01 = g_corner(g, vx, FyBx, x, y + 1, z, 1, 0);
  const T YX10 = g_corner(g, vx, FyBx, x + 1, y, z, 1, 0);
  const T XZ00 = g_corner(g, vz, FxBz, x, y, z, 0, 2), XZ01 = g_corner(g, vz, FxBz, x, y, z + 1, 0, 2);
  const T XZ10 = g_corner(g, vz, FxBz, x + 1, y, z, 0, 2);
  const T ZX00 = g_corner(g, vx, FzBx, x, y, z, 2, 0), ZX01 = g_corner(g, vx, FzBx, x, y, z + 1, 2, 0);
  const T ZX10 = g_corner(g, vx, FzBx, x + 1, y, z, 2, 0);
  const T YZ00 = g_corner(g, vz, FyBz, x, y, z, 1, 2), YZ01 = g_corner(g, vz, FyBz, x, y, z + 1, 1, 2);
  const T YZ10 = g_corner(g, vz, FyBz, x, y + 1, z, 1, 2);
  const T ZY00 = g_corner(g, vy, FzBy, x, y, z, 2, 1), ZY01 = g_corner(g, vy, FzBy, x, y, z + 1, 2, 1);
  const T ZY10 = g_corner(g, vy, FzBy, x, y + 1, z, 2, 1);
  const T dx = to<T>(g.dx), dy = to<T>(g.dy), dz = to<T>(g.dz), half = to<T>(0.5f);
  T pb = to<T>(0.0f);
  pb = pb + half * ((XY01 - XY00) / dy + (XZ01 - XZ00) / dz);
  pb = pb - half * (YX01 - YX00) / dy;
  pb = pb - half * (ZX01 - ZX00) / dz;
  wo[5 * N + o] = wb[5 * N + o] + h * pb;
  pb = to<T>(0.0f);
  pb = pb - half * (XY10 - XY00) / dx;
  pb = pb + half * ((YZ01 - YZ00) / dz + (YX10 - YX00) / dx);
  pb = pb - half * (ZY01 - ZY00) / dz;
  wo[6 * N + o] = wb[6 * N + o] + h * pb;
  pb = to<T>(0.0f);
  pb = pb - half * (XZ10 - XZ00) / dx;
  pb = pb - half * (YZ10 - YZ00) / dy;
  pb = pb + half * ((ZX10 - ZX00) / dx + (ZY10 - ZY00) / dy);
  wo[7 * N + o] = wb[7 * N + o] + h * pb;
}

// Flux divergence, conserved update, primitive recovery with the new face B
// and the Kepler kick (cell fields of wo; its face B come from g_ct_cell).
template <class T, class R>
NMHD_HD void g_prim_cell(const GGrid<R> &g, const T *wb, T *wo, const T *flux, int x, int y, int z, const T &h) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  const int oxp = cell_at(g, x + 1, y, z), oyp = cell_at(g, x, y + 1, z), ozp = cell_at(g, x, y, z + 1);
  const T *Fx = flux, *Fy = flux + 7 * N, *Fz = flux + 14 * N;
  const T dx = to<T>(g.dx), dy = to<T>(g.dy), dz = to<T>(g.dz);
  T pace[5];
  for (int v = 0; v < 5; ++v) {
    T pc = to<T>(0.0f);
    pc = pc + (Fx[v * N + o] - Fx[v * N + oxp]) / dx;
    pc = pc + (Fy[v * N + o] - Fy[v * N + oyp]) / dy;
    pc = pc + (Fz[v * N + o] - Fz[v * N + ozp]) / dz;
    pace[v] = pc;
  }
  const T gm1 = to<T>(g.gamma) - to<T>(1.0f);
  const T rho0 = wb[o], vx0 = wb[N + o], vy0 = wb[2 * N + o], vz0 = wb[3 * N + o], p0 = wb[4 * N + o];
  const T bxl = wb[5 * N + o], bxh = wb[5 * N + oxp];
  const T byl = wb[6 * N + o], byh = wb[6 * N + oyp];
  const T bzl = wb[7 * N + o], bzh = wb[7 * N + ozp];
  const T mx0 = rho0 * vx0, my0 = rho0 * vy0, mz0 = rho0 * vz0;
  const T e0 = p0 / gm1 + to<T>(0.5f) * rho0 * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0) +
               to<T>(0.25f) * (bxl * bxl + bxh * bxh + byl * byl + byh * byh + bzl * bzl + bzh * bzh);
  const T rho = rho0 + h * pace[0];
  const T mx = mx0 + h * pace[1];
  const T my = my0 + h * pace[2];
  const T mz = mz0 + h * pace[3];
  const T ene = e0 + h * pace[4];
  const T bx0 = wo[5 * N + o], bx1 = wo[5 * N + oxp];
  const T by0 = wo[6 * N + o], by1 = wo[6 * N + oyp];
  const T bz0 = wo[7 * N + o], bz1 = wo[7 * N + ozp];
  T vxo = mx / rho, vyo = my / rho, vzo = mz / rho;
  const T eint = ene - to<T>(0.5f) * (mx * mx + my * my + mz * mz) / rho -
                 to<T>(0.25f) * (bx0 * bx0 + bx1 * bx1 + by0 * by0 + by1 * by1 + bz0 * bz0 + bz1 * bz1);
  const T po = eint * gm1;
  if (g.shear) {
    const T ax = to<T>(-2.0f) * to<T>(g.omega) * vyo;
    const T ay = to<T>(2.0f) * to<T>(g.omega) * vxo +
                 to<T>(R(2.0f) * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((R)y + R(0.5f))));
    vxo = vxo + h * ax;
    vyo = vyo + h * ay;
    vzo = vzo + h * to<T>(0.0f);
  }
  wo[o] = rho;
  wo[N + o] = vxo;
  wo[2 * N + o] = vyo;
  wo[3 * N + o] = vzo;
  wo[4 * N + o] = po;
}

// Shearing-periodic Y-margin fill, one item (sx, sy, sz) with sy < margin_y
// (communicate_gather/scatter_kernel_y with relative_displacement).
template <class R>
NMHD_HD void shear_shift(const GGrid<R> &g, double time, int &dint, R &f) {
  const double d0 = 0.0 + time * g.rel_vel;
  const int fold = (int)floor(d0 / (double)g.extent_x);
  const double d1 = d0 - (double)((R)fold * g.extent_x);
  dint = (int)floor(d1 / (double)g.dx);
  f = (R)(d1 / (double)g.dx - dint);
}

template <class T, class R>
NMHD_HD void g_fill_y_item(const GGrid<R> &g, double time, T *w, int idx) {
  const int M = g.my;
  const int sx = idx % g.sx;
  const int sy = (idx / g.sx) % M;
  const int sz = idx / (g.sx * M);
  int dint;
  R f;
  shear_shift(g, time, dint, f);
  const R rv = (R)g.rel_vel;
  const int inc_x = wrapc((sx + dint) % g.sx, g.sx);
  const int dec_x = wrapc((sx - dint - 1) % g.sx, g.sx);
  const size_t N = (size_t)g.n;
  const int src_inc = (sz * g.sy + (g.sy - 2 * M + sy)) * g.sx + inc_x;
  const int src_dec = (sz * g.sy + (M + sy)) * g.sx + dec_x;
  const int dst_lo = (sz * g.sy + sy) * g.sx + sx;
  const int dst_hi = (sz * g.sy + (g.sy - M + sy)) * g.sx + sx;
  const T omf = to<T>(R(1.0f) - f), ff = to<T>(f);
  for (int v = 0; v < 8; ++v) {
    const T vi = w[v * N + src_inc];
    const T vd = w[v * N + src_dec];
    T bi = omf * vi + ff * vi;
    T bd = ff * vd + omf * vd;
    if (v == 1) {
      bi = bi - to<T>(rv);
      bd = bd + to<T>(rv);
    }
    w[v * N + dst_lo] = bi;
    if (!(v == 6 && sy == 0)) w[v * N + dst_hi] = bd;
  }
}

// Plain periodic Z-margin copy, one item of the sx*sy*mz plane block.
template <class T, class R>
NMHD_HD void g_fill_z_item(const GGrid<R> &g, T *w, int idx) {
  const size_t n = (size_t)g.n, unit = (size_t)g.sx * g.sy * g.mz;
  for (int v = 0; v < 8; ++v) {
    T *var = w + v * n;
    const T lo = var[n - 2 * unit + idx];
    const T hi = var[unit + idx];
    var[idx] = lo;
    var[n - unit + idx] = hi;
  }
}

// -<Bx By> of one interior cell at the cell centre (the diagnostics' Maxwell
// stress), in FP64 (or its dual).
template <class T>
struct Wide64 { typedef double type; };
template <class R>
struct Wide64<Dual<R>> { typedef Dual<double> type; };

template <class T, class R>
NMHD_HD typename Wide64<T>::type g_stress_cell(const GGrid<R> &g, const T *w, int x, int y, int z) {
  typedef typename Wide64<T>::type D;
  const size_t N = (size_t)g.n;
  if (y < g.my || y >= g.sy - g.my || z < g.mz || z >= g.sz - g.mz) return to<D>(0.0);
  const int o = cell_at(g, x, y, z);
  const D bxl = to<D>(w[5 * N + o]), bxh = to<D>(w[5 * N + cell_at(g, x + 1, y, z)]);
  const D byl = to<D>(w[6 * N + o]), byh = to<D>(w[6 * N + cell_at(g, x, y + 1, z)]);
  return -(to<D>(0.25) * (bxl + bxh) * (byl + byh));
}

// ---------------------------------------------------------------------------
// Adjoint.  Scratch layout (N values per field):
//   lamU  5 fields: adjoint of the updated conserved state (rho, m_x, m_y,
//         m_z, E) of the stage, which is also that of the conserved state
//         before it;
//   lamE  1 field: adjoint of the internal energy;
//   lamBn 3 fields: adjoint of the new face B (x, y, z);
//   face  30 fields, one face axis at a time: for the 7 reconstructed
//         variables (rho, v_n, v_t1, v_t2, p, B_t1, B_t2 averages) the
//         contributions to the 4 cells the face's reconstruction reads
//         (4*v + k: cell face - 2 + k), then the half-kick (28) and the normal
//         face field (29);
//   lamBc 3 fields: adjoint of the cell-centred transverse B averages.

template <class R>
NMHD_HD void a_prim_cell(const GGrid<R> &g, const R *wb, const R *wo, const R *lout, R *lamU, R *lamE, R *lb,
                         int x, int y, int z, R h) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  // the linearisation point, the updated conserved state, from the stage's
  // output: its density is the updated density, its velocity m/rho after the
  // Kepler kick, which is undone here (vx' = vx - c vy, vy' = vy + c vx + h T,
  // c = 2 omega h)
  const R gm1 = g.gamma - R(1.0f);
  const R rho0 = wb[o], vx0 = wb[N + o], vy0 = wb[2 * N + o], vz0 = wb[3 * N + o];
  const R rho = wo[o];
  R vx = wo[N + o], vy = wo[2 * N + o];
  const R vz = wo[3 * N + o];
  if (g.shear) {
    const R c = R(2.0f) * g.omega * h;
    const R tidal = h * (R(2.0f) * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((R)y + R(0.5f))));
    const R vyk = vy - tidal, id = R(1) / (R(1) + c * c);
    const R vxp = (vx + c * vyk) * id;
    vy = (vyk - c * vx) * id;
    vx = vxp;
  }
  const R mx = rho * vx, my = rho * vy, mz = rho * vz;
  R l_vx = lout[N + o], l_vy = lout[2 * N + o];
  const R l_vz = lout[3 * N + o];
  if (g.shear) {
    // vx' = vx - 2 omega h vy,  vy' = vy + 2 omega h vx + const
    const R c = R(2.0f) * g.omega * h;
    const R lx = l_vx + c * l_vy;
    const R ly = l_vy - c * l_vx;
    l_vx = lx;
    l_vy = ly;
  }
  const R l_eint = gm1 * lout[4 * N + o];
  const R ir = R(1) / rho;
  const R l_mx = (l_vx - l_eint * mx) * ir;
  const R l_my = (l_vy - l_eint * my) * ir;
  const R l_mz = (l_vz - l_eint * mz) * ir;
  const R l_rho = lout[o] + (l_eint * R(0.5f) * (mx * mx + my * my + mz * mz) -
                             (l_vx * mx + l_vy * my + l_vz * mz)) * (ir * ir);
  const R l_ene = l_eint;
  lamU[o] = l_rho;
  lamU[N + o] = l_mx;
  lamU[2 * N + o] = l_my;
  lamU[3 * N + o] = l_mz;
  lamU[4 * N + o] = l_ene;
  lamE[o] = l_eint;
  // conserved state before the stage from the base primitives
  lb[o] = fmaa(l_ene * R(0.5f), (vx0 * vx0 + vy0 * vy0 + vz0 * vz0), fmaa(l_mz, vz0, fmaa(l_my, vy0, fmaa(l_mx, vx0, lb[o] + l_rho))));
  lb[N + o] += (l_mx + l_ene * vx0) * rho0;
  lb[2 * N + o] += (l_my + l_ene * vy0) * rho0;
  lb[3 * N + o] += (l_mz + l_ene * vz0) * rho0;
  lb[4 * N + o] += l_ene * (R(1) / gm1);
}

template <class R>
NMHD_HD void a_bface_cell(const GGrid<R> &g, const R *wb, const R *wo, const R *lout, const R *lamU, const R *lamE,
                          R *lamBn, R *lb, int x, int y, int z) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  for (int a = 0; a < 3; ++a) {
    const int om = shifted(g, x, y, z, a, -1);
    const size_t fb = (size_t)(5 + a) * N;
    const R l = lout[fb + o] - R(0.5f) * wo[fb + o] * (lamE[o] + lamE[om]);
    lamBn[a * N + o] = l;
    lb[fb + o] += l + R(0.5f) * wb[fb + o] * (lamU[4 * N + o] + lamU[4 * N + om]);
  }
}

// Periodic neighbour offsets of one cell, computed once per thread: the
// address of (x+i, y+j, z+k), |i|, |j|, |k| <= 3, is o + d[0][i+3] + d[1][j+3]
// + d[2][k+3] (the axes wrap independently, so displacements along different
// axes add).  With the axis a template parameter the table stays in registers.
struct Nbr {
  int o;
  int d[3][7];
};

template <class R>
NMHD_HD Nbr make_nbr(const GGrid<R> &g, int x, int y, int z) {
  Nbr n;
  n.o = (z * g.sy + y) * g.sx + x;
  const int sxy = g.sx * g.sy;
#pragma unroll
  for (int k = -3; k <= 3; ++k) {
    n.d[0][k + 3] = wrapc(x + k, g.sx) - x;
    n.d[1][k + 3] = (wrapc(y + k, g.sy) - y) * g.sx;
    n.d[2][k + 3] = (wrapc(z + k, g.sz) - z) * sxy;
  }
  return n;
}

// face_input for the lower AX-face, addresses from the offset table (the same
// arithmetic as face_input).
// Minbee choices of one reconstruction (same operations as reconstruct4_g),
// packed as cl | cr << 2 (0: zero slope, 1: first difference, 2: second).
template <class R>
NMHD_HD unsigned mm_choices(R x0, R x1, R x2, R x3) {
  const R d01 = x1 - x0, d12 = x2 - x1, d23 = x3 - x2;
  const unsigned cl = d01 * d12 <= R(0) ? 0u : (gabs(d01) < gabs(d12) ? 1u : 2u);
  const unsigned cr = d12 * d23 <= R(0) ? 0u : (gabs(d12) < gabs(d23) ? 1u : 2u);
  return cl | (cr << 2);
}

template <int AX, class T, class R>
NMHD_HD void face_input_nb(const GGrid<R> &g, const T *w, const Nbr &nb, int y, const T &h, HState<T> &in,
                           T &bn, unsigned *choices = nullptr) {
  constexpr int E1 = (AX + 1) % 3, E2 = (AX + 2) % 3;
  const size_t N = (size_t)g.n;
  int c[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) c[t] = nb.o + nb.d[AX][t + 1];
  const int t1 = nb.d[E1][4], t2 = nb.d[E2][4];
  const T *rho = w, *p = w + 4 * N;
  const T *vn = w + (1 + AX) * N, *v1 = w + (1 + E1) * N, *v2 = w + (1 + E2) * N;
  const T *b1 = w + (5 + E1) * N, *b2 = w + (5 + E2) * N;
  T bc1[4], bc2[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    bc1[t] = to<T>(0.5f) * (b1[c[t]] + b1[c[t] + t1]);
    bc2[t] = to<T>(0.5f) * (b2[c[t]] + b2[c[t] + t2]);
  }
  if (g.order2) {
    reconstruct4_g(rho[c[0]], rho[c[1]], rho[c[2]], rho[c[3]], in.dl, in.dr);
    reconstruct4_g(vn[c[0]], vn[c[1]], vn[c[2]], vn[c[3]], in.ul, in.ur);
    reconstruct4_g(v1[c[0]], v1[c[1]], v1[c[2]], v1[c[3]], in.vl, in.vr);
    reconstruct4_g(v2[c[0]], v2[c[1]], v2[c[2]], v2[c[3]], in.wl, in.wr);
    reconstruct4_g(p[c[0]], p[c[1]], p[c[2]], p[c[3]], in.pl, in.pr);
    reconstruct4_g(bc1[0], bc1[1], bc1[2], bc1[3], in.byl, in.byr);
    reconstruct4_g(bc2[0], bc2[1], bc2[2], bc2[3], in.bzl, in.bzr);
    if (choices) {
      *choices = mm_choices(val(rho[c[0]]), val(rho[c[1]]), val(rho[c[2]]), val(rho[c[3]])) |
                 mm_choices(val(vn[c[0]]), val(vn[c[1]]), val(vn[c[2]]), val(vn[c[3]])) << 4 |
                 mm_choices(val(v1[c[0]]), val(v1[c[1]]), val(v1[c[2]]), val(v1[c[3]])) << 8 |
                 mm_choices(val(v2[c[0]]), val(v2[c[1]]), val(v2[c[2]]), val(v2[c[3]])) << 12 |
                 mm_choices(val(p[c[0]]), val(p[c[1]]), val(p[c[2]]), val(p[c[3]])) << 16 |
                 mm_choices(val(bc1[0]), val(bc1[1]), val(bc1[2]), val(bc1[3])) << 20 |
                 mm_choices(val(bc2[0]), val(bc2[1]), val(bc2[2]), val(bc2[3])) << 24;
    }
  } else {
    in.dl = rho[c[1]]; in.dr = rho[c[2]];
    in.ul = vn[c[1]]; in.ur = vn[c[2]];
    in.vl = v1[c[1]]; in.vr = v1[c[2]];
    in.wl = v2[c[1]]; in.wr = v2[c[2]];
    in.pl = p[c[1]]; in.pr = p[c[2]];
    in.byl = bc1[1]; in.byr = bc1[2];
    in.bzl = bc2[1]; in.bzr = bc2[2];
    if (choices) *choices = 0u;  // left = x1, right = x2: the zero-slope weights
  }
  if (g.shear) {
    T acc;
    if (AX == 0) {
      const T vY = to<T>(0.5f) * (w[2 * N + c[1]] + w[2 * N + c[2]]);
      acc = to<T>(-2.0f) * to<T>(g.omega) * vY;
    } else if (AX == 1) {
      const T vX = to<T>(0.5f) * (w[N + c[1]] + w[N + c[2]]);
      acc = to<T>(2.0f) * to<T>(g.omega) * vX +
            to<T>(R(2.0f) * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((R)y + R(0.5f))));
    } else {
      acc = to<T>(R(0));
    }
    const T mbv = to<T>(0.5f) * h * acc;
    in.ul = in.ul + mbv;
    in.ur = in.ur + mbv;
  }
  bn = w[(5 + AX) * N + c[2]];
}

// Adjoint of the flux F_A(B_B) at the cell's lower A-face: the CT transpose.
// The corner value C = F_A(B_B) at an edge e is F[e - B] (4-cell wind sum of
// v_B > 0), F[e] (< 0) or their mean; it enters the face-B updates as
//   dB_A[o] = +h/2 (C[o+B] - C[o]) / d_B,   dB_B[o] = -h/2 (C[o+A] - C[o]) / d_A
// in every family (XY, YX, XZ, ZX, YZ, ZY).  F at the cell's face enters the
// corners at the cell's edge (as F[e]) and one step up B (as F[e - B]).
template <int A, int B, class R>
NMHD_HD R ct_flux_adj_nb(const GGrid<R> &g, const R *win, const R *lamBn, const Nbr &nb, R h) {
  const size_t N = (size_t)g.n;
  const R *vb = win + (1 + B) * N;
  const R *lA = lamBn + A * N, *lB = lamBn + B * N;
  const R ca = h * R(0.5f) * inv_spacing(g, B);
  const R cb = h * R(0.5f) * inv_spacing(g, A);
  R acc = R(0);
#pragma unroll
  for (int db = 0; db < 2; ++db) {  // edge at displacement db along B (0 or +1)
    const int e = nb.o + nb.d[B][db + 3];
    const int eb = nb.o + nb.d[B][db + 2];
    const int ea = nb.o + nb.d[A][2] + nb.d[B][db + 3];
    const int eab = nb.o + nb.d[A][2] + nb.d[B][db + 2];
    const R wind = vb[e] + vb[eb] + vb[ea] + vb[eab];
    // weight of this face's F in the corner: F[e] for db = 0, F[e - B] for db = 1
    const R wgt = db == 0 ? (wind > R(0) ? R(0) : (wind < R(0) ? R(1) : R(0.5f)))
                          : (wind > R(0) ? R(1) : (wind < R(0) ? R(0) : R(0.5f)));
    const R lam_c = ca * (lA[eb] - lA[e]) - cb * (lB[ea] - lB[e]);
    acc = fmaa(wgt, lam_c, acc);
  }
  return acc;
}

// Adjoint of the lower AX-face flux of the cell: flux-divergence and CT
// transposes give the adjoint of its 7 fluxes, the HLLD adjoint that of the
// Riemann input, stored at face + (15*AX + k)*N.
template <int AX, class R>
NMHD_HD void a_flux_face(const GGrid<R> &g, const R *win, const R *lamBn, const R *lamU, R *face, int x, int y,
                         int z, R h) {
  constexpr int E1 = (AX + 1) % 3, E2 = (AX + 2) % 3;
  const size_t N = (size_t)g.n;
  const Nbr nb = make_nbr(g, x, y, z);
  const int o = nb.o, om = o + nb.d[AX][2];
  const R c = h * inv_spacing(g, AX);
  R lfa[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) lfa[k] = c * (lamU[k * N + o] - lamU[k * N + om]);
  R lf[7];
  lf[0] = lfa[0];
  lf[1] = lfa[1 + AX];
  lf[2] = lfa[1 + E1];
  lf[3] = lfa[1 + E2];
  lf[4] = lfa[4];
  lf[5] = ct_flux_adj_nb<AX, E1>(g, win, lamBn, nb, h);
  lf[6] = ct_flux_adj_nb<AX, E2>(g, win, lamBn, nb, h);
  HState<R> in;
  R bn;
  unsigned ch;
  face_input_nb<AX>(g, win, nb, y, h, in, bn, &ch);
  HState<R> ls;
  R lbn;
  hlld_adjoint(g.gamma, bn, in, lf, ls, lbn);
  // Transpose of the reconstruction of each variable at this face, split by
  // the four cells x0..x3 (= face - 2 .. face + 1 along AX) it reads:
  // left = x1 + d1/2 with d1 = 0 | x1 - x0 | x2 - x1, right = x2 - d2/2 with
  // d2 = 0 | x2 - x1 | x3 - x2 (the choice frozen at the forward's).
  const R lL[7] = {ls.dl, ls.ul, ls.vl, ls.wl, ls.pl, ls.byl, ls.bzl};
  const R lR[7] = {ls.dr, ls.ur, ls.vr, ls.wr, ls.pr, ls.byr, ls.bzr};
  R *fo = face + o;
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    const unsigned cl = (ch >> (4 * v)) & 3u, cr = (ch >> (4 * v + 2)) & 3u;
    const R a = lL[v], b = lR[v];
    R t0 = R(0), t1 = R(0), t2 = R(0), t3 = R(0);
    if (cl == 0u) { t1 += a; }
    else if (cl == 1u) { t0 -= R(0.5f) * a; t1 += R(1.5f) * a; }
    else { t1 += R(0.5f) * a; t2 += R(0.5f) * a; }
    if (cr == 0u) { t2 += b; }
    else if (cr == 1u) { t1 += R(0.5f) * b; t2 += R(0.5f) * b; }
    else { t2 += R(1.5f) * b; t3 -= R(0.5f) * b; }
    fo[(4 * v) * N] = t0;
    fo[(4 * v + 1) * N] = t1;
    fo[(4 * v + 2) * N] = t2;
    fo[(4 * v + 3) * N] = t3;
  }
  fo[28 * N] = ls.ul + ls.ur;  // adjoint of the face half-kick
  fo[29 * N] = lbn;            // adjoint of the normal face field
}

// Gather of the AX-face reconstruction transposes at cell c: each variable of
// the cell receives the contributions of faces c + 2, c + 1, c, c - 1 (where
// it is x0, x1, x2, x3), written by a_flux_face for this axis; the cell-centred
// transverse B averages go to lamBc, the face half-kick to v_y (AX 0) or v_x
// (AX 1), the normal field of face c to B_AX.  Called for AX = 0, 1, 2 in
// turn, each after a_flux_face of the same axis; lin and lamBc accumulate.
template <int AX, class R>
NMHD_HD void a_recon_face(const GGrid<R> &g, const R *face, R *lin, R *lamBc, int x, int y, int z, R h) {
  constexpr int E1 = (AX + 1) % 3, E2 = (AX + 2) % 3;
  const size_t N = (size_t)g.n;
  const Nbr nb = make_nbr(g, x, y, z);
  const int o = nb.o;
  int f[4];  // face of which this cell is x_k
#pragma unroll
  for (int k = 0; k < 4; ++k) f[k] = o + nb.d[AX][5 - k];
  R lv[7];
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    R acc = R(0);
#pragma unroll
    for (int k = 0; k < 4; ++k) acc += face[(4 * v + k) * N + f[k]];
    lv[v] = acc;
  }
  if (g.shear && AX < 2) {
    // mbv(f) = h/2 * acc(f); acc takes the mean of the two cells of face f,
    // d acc / d v = -2 omega (AX 0, v_y) or +2 omega (AX 1, v_x)
    const R lm = face[28 * N + o] + face[28 * N + f[1]];
    lv[AX == 0 ? 2 : 3] += R(0.5f) * h * (AX == 0 ? -g.omega : g.omega) * lm;
  }
  lin[o] += lv[0];
  lin[(1 + AX) * N + o] += lv[1];
  lin[(1 + E1) * N + o] += lv[2];
  lin[(1 + E2) * N + o] += lv[3];
  lin[4 * N + o] += lv[4];
  lamBc[E1 * N + o] += lv[5];
  lamBc[E2 * N + o] += lv[6];
  lin[(5 + AX) * N + o] += face[29 * N + o];
}

template <class R>
NMHD_HD void a_bc_cell(const GGrid<R> &g, const R *lamBc, R *lin, int x, int y, int z) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  for (int c = 0; c < 3; ++c)
    lin[(5 + c) * N + o] += R(0.5f) * (lamBc[c * N + o] + lamBc[c * N + shifted(g, x, y, z, c, -1)]);
}

// Transpose of g_fill_z_item (one item; margins read, added to their sources
// and cleared by the same thread).
template <class R>
NMHD_HD void a_fill_z_item(const GGrid<R> &g, R *lam, int idx) {
  const size_t n = (size_t)g.n, unit = (size_t)g.sx * g.sy * g.mz;
  for (int v = 0; v < 8; ++v) {
    R *var = lam + v * n;
    const R lo = var[idx], hi = var[n - unit + idx];
    var[idx] = R(0);
    var[n - unit + idx] = R(0);
    var[n - 2 * unit + idx] += lo;
    var[unit + idx] += hi;
  }
}

// Transpose of g_fill_y_item, gathered at the source: item (xs, sy, sz)
// covers, for all 8 fields, the source cells (xs, Sy-2M+sy, sz) (-> bottom
// margin row sy) and (xs, M+sy, sz) (-> top margin row Sy-M+sy).  Each margin
// cell is the image of exactly one item, which clears it after reading; margin
// and source rows are disjoint, so every load is issued before any store.  With
// exactly M interior rows the two source cells coincide and take both
// contributions, bottom first.  dint and f are shear_shift() of the step's time.
template <class R>
NMHD_HD void a_fill_y_item(const GGrid<R> &g, int dint, R f, R *lam, int idx) {
  const int M = g.my;
  const size_t N = (size_t)g.n;
  const int xs = idx % g.sx;
  const int sy = (idx / g.sx) % M;
  const int sz = idx / (g.sx * M);
  const R coef = (R(1.0f) - f) + f;  // d/dv of (1-f) v + f v
  const int sx_lo = wrapc((xs - dint) % g.sx, g.sx);      // (sx_lo + dint) mod Sx = xs
  const int sx_hi = wrapc((xs + dint + 1) % g.sx, g.sx);  // (sx_hi - dint - 1) mod Sx = xs
  const int src_inc = (sz * g.sy + (g.sy - 2 * M + sy)) * g.sx + xs;
  const int src_dec = (sz * g.sy + (M + sy)) * g.sx + xs;
  const int dst_lo = (sz * g.sy + sy) * g.sx + sx_lo;
  const int dst_hi = (sz * g.sy + (g.sy - M + sy)) * g.sx + sx_hi;
  R llo[8], lhi[8], ai[8], ad[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    llo[v] = lam[v * N + dst_lo];
    lhi[v] = (v == 6 && sy == 0) ? R(0) : lam[v * N + dst_hi];  // By of row Sy-M is interior
    ai[v] = lam[v * N + src_inc];
    ad[v] = lam[v * N + src_dec];
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    lam[v * N + dst_lo] = R(0);
    if (!(v == 6 && sy == 0)) lam[v * N + dst_hi] = R(0);
    if (src_inc == src_dec) {
      lam[v * N + src_inc] = fmaa(coef, lhi[v], fmaa(coef, llo[v], ai[v]));
    } else {
      lam[v * N + src_inc] = fmaa(coef, llo[v], ai[v]);
      lam[v * N + src_dec] = fmaa(coef, lhi[v], ad[v]);
    }
  }
}

// Gradient of s * sum over interior cells of -(Bx By at the cell centre)
// with respect to the face fields of cell (x, y, z), added to lam.
template <class R>
NMHD_HD void a_stress_cell(const GGrid<R> &g, const R *w, R *lam, int x, int y, int z, double s) {
  const size_t N = (size_t)g.n;
  const int o = cell_at(g, x, y, z);
  auto inner = [&](int yy, int zz) {
    return yy >= g.my && yy < g.sy - g.my && zz >= g.mz && zz < g.sz - g.mz;
  };
  double gx = 0.0, gy = 0.0;
  // cells using Bx[o]: (x, y, z) as its low face, (x-1, y, z) as its high face
  for (int k = 0; k < 2; ++k) {
    const int cx = x - k;
    if (!inner(y, z)) break;
    const double byl = (double)w[6 * N + cell_at(g, cx, y, z)], byh = (double)w[6 * N + cell_at(g, cx, y + 1, z)];
    gx = fmaa(-0.25, (byl + byh), gx);
  }
  for (int k = 0; k < 2; ++k) {
    const int cy = wrapc(y - k, g.sy);
    if (!inner(cy, z)) continue;
    const double bxl = (double)w[5 * N + cell_at(g, x, cy, z)], bxh = (double)w[5 * N + cell_at(g, x + 1, cy, z)];
    gy = fmaa(-0.25, (bxl + bxh), gy);
  }
  lam[5 * N + o] += (R)(s * gx);
  lam[6 * N + o] += (R)(s * gy);
}

}  // namespace ad
}  // namespace nmhd
