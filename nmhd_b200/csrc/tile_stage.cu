// Tiled stage kernels (v2) of the B200 ideal-MHD time step, sm_100a.
//
// One RK stage = two kernels over the whole box, each a 2.5-D march: a CTA
// owns a 32 x TY column of cells in x-y and walks a chunk of z planes, keeping
// a ring of three planes (with a 2-cell x-y halo) in shared memory.
//
//  k_tile_flux   reconstruction + HLLD on the x-, y- and z-faces of its cells
//                (calc_flux_kernel<X,Y,Z>, src/library/mhd_solver.inlrb:562-636),
//                the flux divergence of rho, m, E (add_flux_kernel :689-693),
//                and the conserved update U = U_bef + dt*pace (to_conserved,
//                add_pace/update :762-835).  Writes 5 conserved values and the
//                6 face fluxes of B the constrained transport needs.  Every
//                face is solved once; only one extra x-face per row and one
//                extra y-face per column of the tile are solved twice.
//  k_tile_ct     corner EMFs and the face-B update (:641-714), primitive
//                recovery (:779-795), the Kepler kick (:837-848) and, in the
//                final stage, the CFL reduction for the next step and the clock
//                update (:496-521, 870-901, 981).
//
// Arithmetic is the reference's, operation by operation (mhd_math.cuh); the
// file is compiled with -fmad=false.
#include "mhd_math.cuh"
#include "step.cuh"

namespace nmhd {

namespace {

constexpr int TX = 32;

__device__ __forceinline__ int wrapi(int v, int s) {
  while (v < 0) v += s;
  while (v >= s) v -= s;
  return v;
}

__device__ __forceinline__ float dt_of(const StepCtl *c, bool *last) {
  if (c->dt_seq) {
    if (last) *last = false;
    return c->dt_seq[c->generation - c->dt_seq_base];
  }
  const float cmin = __uint_as_float(c->cfl_cur);
  float dt = fminf(c->goal, cmin);
  const double next_time = c->time + (double)dt;
  const bool l = next_time > (double)c->goal;
  if (l) dt = (float)((double)c->goal - c->time);
  if (last) *last = l;
  return dt;
}

__device__ __forceinline__ const float *pick(const StepCtl *c, int sel, const float *w0, const float *w1,
                                             const float *wp) {
  if (sel == 2) return wp;
  return (sel == 0) == (c->parity == 0) ? w0 : w1;
}

__device__ __forceinline__ float kepler_y(const GridParams &g, int y) {
  return g.corner_y + g.dy * ((float)y + 0.5f);
}

// Load plane z of the 8 primitive fields into a (TY+2H) x (32+2H) slot (halo H),
// coordinates wrapped periodically.
// Fields 0..NA-1 come from base_a, the rest from base_b (each Sx*Sy*Sz floats).
template <int TY, int H, int NF, int NA>
__device__ __forceinline__ void load_plane(float *slot, const float *base_a, const float *base_b,
                                           const GridParams &g, int x0, int y0, int z) {
  constexpr int PX = TX + 2 * H, PY = TY + 2 * H, PLANE = PX * PY;
  const int zw = wrapi(z, g.sz);
  const int tid = threadIdx.y * TX + threadIdx.x;
  constexpr int NT = TX * TY;
  for (int e = tid; e < NF * PLANE; e += NT) {
    const int f = e / PLANE;
    const int rem = e - f * PLANE;
    const int r = rem / PX;
    const int c = rem - r * PX;
    const int yw = wrapi(y0 - H + r, g.sy);
    const int xw = wrapi(x0 - H + c, g.sx);
    const float *src = f < NA ? base_a + (size_t)f * g.n : base_b + (size_t)(f - NA) * g.n;
    slot[e] = __ldg(src + ((size_t)zw * g.sy + yw) * g.sx + xw);
  }
}

// Primitive fields (density, vx, vy, vz, pressure, Bx, By, Bz) in a plane slot.
enum { F_RHO = 0, F_VX = 1, F_VY = 2, F_VZ = 3, F_P = 4, F_BX = 5, F_BY = 6, F_BZ = 7 };

// HLLD input for the face between cells c-1 and c along x or y, built from the
// smem slot (halo 2).  AX = 0: x-face at (row r, col c); AX = 1: y-face.
// `up` is the slot of the plane above (its B_z is the upper z-face of this plane).
template <int AX, int TY>
__device__ __forceinline__ void xy_face(const GridParams &g, const float *slot, const float *up, int r,
                                        int c, int yface, float dt, float out[7]) {
  constexpr int PX = TX + 4, PLANE = PX * (TY + 4);
  // smem index of stencil cell t (t = 0..3 -> offsets -2..+1 along AX)
  auto at = [&](int t) {
    return AX == 0 ? (r + 2) * PX + (c + t) : (r + t) * PX + (c + 2);
  };
  const float *rho = slot + F_RHO * PLANE, *p = slot + F_P * PLANE;
  const float *vn = slot + (AX == 0 ? F_VX : F_VY) * PLANE;
  const float *vt1 = slot + (AX == 0 ? F_VY : F_VZ) * PLANE;
  const float *vt2 = slot + (AX == 0 ? F_VZ : F_VX) * PLANE;
  // transverse B (t1, t2) = (By, Bz) for x-faces, (Bz, Bx) for y-faces
  float b1[4], b2[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int i = at(t);
    if (AX == 0) {
      b1[t] = 0.5f * (slot[F_BY * PLANE + i] + slot[F_BY * PLANE + i + PX]);
      b2[t] = 0.5f * (slot[F_BZ * PLANE + i] + up[F_BZ * PLANE + i]);
    } else {
      b1[t] = 0.5f * (slot[F_BZ * PLANE + i] + up[F_BZ * PLANE + i]);
      b2[t] = 0.5f * (slot[F_BX * PLANE + i] + slot[F_BX * PLANE + i + 1]);
    }
  }
  HlldIn s;
  if (g.order2) {
    reconstruct4(rho[at(0)], rho[at(1)], rho[at(2)], rho[at(3)], s.dl, s.dr);
    reconstruct4(vn[at(0)], vn[at(1)], vn[at(2)], vn[at(3)], s.ul, s.ur);
    reconstruct4(vt1[at(0)], vt1[at(1)], vt1[at(2)], vt1[at(3)], s.vl, s.vr);
    reconstruct4(vt2[at(0)], vt2[at(1)], vt2[at(2)], vt2[at(3)], s.wl, s.wr);
    reconstruct4(p[at(0)], p[at(1)], p[at(2)], p[at(3)], s.pl, s.pr);
    reconstruct4(b1[0], b1[1], b1[2], b1[3], s.byl, s.byr);
    reconstruct4(b2[0], b2[1], b2[2], b2[3], s.bzl, s.bzr);
  } else {
    s.dl = rho[at(1)]; s.dr = rho[at(2)];
    s.ul = vn[at(1)]; s.ur = vn[at(2)];
    s.vl = vt1[at(1)]; s.vr = vt1[at(2)];
    s.wl = vt2[at(1)]; s.wr = vt2[at(2)];
    s.pl = p[at(1)]; s.pr = p[at(2)];
    s.byl = b1[1]; s.byr = b1[2];
    s.bzl = b2[1]; s.bzr = b2[2];
  }
  if (g.shear) {
    float acc;
    if (AX == 0) {
      const float vY = 0.5f * (slot[F_VY * PLANE + at(1)] + slot[F_VY * PLANE + at(2)]);
      acc = -2.0f * g.omega * vY;
    } else {
      const float vX = 0.5f * (slot[F_VX * PLANE + at(1)] + slot[F_VX * PLANE + at(2)]);
      acc = 2.0f * g.omega * vX + 2.0f * g.q * (g.omega * g.omega) * kepler_y(g, yface);
    }
    const float mbv = 0.5f * dt * acc;
    s.ul += mbv;
    s.ur += mbv;
  }
  const float bn = slot[(AX == 0 ? F_BX : F_BY) * PLANE + at(2)];
  float f[7];
  hlld_flux(g.gamma, bn, s, f);
  // momentum flux components (normal, t1, t2) -> (x, y, z)
  out[0] = f[0];
  out[1] = AX == 0 ? f[1] : f[3];
  out[2] = AX == 0 ? f[2] : f[1];
  out[3] = AX == 0 ? f[3] : f[2];
  out[4] = f[4];
  out[5] = f[5];
  out[6] = f[6];
}

// Per-column reconstruction inputs of one plane for the z-face solve:
// rho, vz, vx, vy, p, <Bx>, <By> (normal = z, t1 = x, t2 = y).
struct ZCol {
  float d, vn, v1, v2, p, b1, b2;
};

template <int TY>
__device__ __forceinline__ ZCol zcol(const float *slot, int r, int c) {
  constexpr int PX = TX + 4, PLANE = PX * (TY + 4);
  const int i = (r + 2) * PX + (c + 2);
  ZCol z;
  z.d = slot[F_RHO * PLANE + i];
  z.vn = slot[F_VZ * PLANE + i];
  z.v1 = slot[F_VX * PLANE + i];
  z.v2 = slot[F_VY * PLANE + i];
  z.p = slot[F_P * PLANE + i];
  z.b1 = 0.5f * (slot[F_BX * PLANE + i] + slot[F_BX * PLANE + i + 1]);
  z.b2 = 0.5f * (slot[F_BY * PLANE + i] + slot[F_BY * PLANE + i + PX]);
  return z;
}

__device__ __forceinline__ void z_face(const GridParams &g, const ZCol &a, const ZCol &b, const ZCol &c,
                                       const ZCol &d, float bn, float dt, float out[7]) {
  HlldIn s;
  if (g.order2) {
    reconstruct4(a.d, b.d, c.d, d.d, s.dl, s.dr);
    reconstruct4(a.vn, b.vn, c.vn, d.vn, s.ul, s.ur);
    reconstruct4(a.v1, b.v1, c.v1, d.v1, s.vl, s.vr);
    reconstruct4(a.v2, b.v2, c.v2, d.v2, s.wl, s.wr);
    reconstruct4(a.p, b.p, c.p, d.p, s.pl, s.pr);
    reconstruct4(a.b1, b.b1, c.b1, d.b1, s.byl, s.byr);
    reconstruct4(a.b2, b.b2, c.b2, d.b2, s.bzl, s.bzr);
  } else {
    s.dl = b.d; s.dr = c.d; s.ul = b.vn; s.ur = c.vn; s.vl = b.v1; s.vr = c.v1;
    s.wl = b.v2; s.wr = c.v2; s.pl = b.p; s.pr = c.p; s.byl = b.b1; s.byr = c.b1;
    s.bzl = b.b2; s.bzr = c.b2;
  }
  if (g.shear) {
    const float mbv = 0.5f * dt * 0.0f;  // no vertical acceleration
    s.ul += mbv;
    s.ur += mbv;
  }
  float f[7];
  hlld_flux(g.gamma, bn, s, f);
  // momentum flux components (normal z, t1 x, t2 y) -> (x, y, z)
  out[0] = f[0];
  out[1] = f[2];
  out[2] = f[3];
  out[3] = f[1];
  out[4] = f[4];
  out[5] = f[5];
  out[6] = f[6];
}

// ---------------------------------------------------------------------------
template <int TY>
__global__ void __launch_bounds__(TX *TY) k_tile_flux(GridParams g, const StepCtl *ctl, const float *w0,
                                                      const float *w1, const float *wp,
                                                      float *__restrict__ unew, float *__restrict__ bflux,
                                                      int in_sel, int half, int zc) {
  constexpr int PX = TX + 4, PY = TY + 4, PLANE = PX * PY, SLOT = 8 * PLANE;
  extern __shared__ float sm[];
  float *ring = sm;                          // [3][8][PY][PX]
  float *fxs = ring + 3 * SLOT;              // [5][TY][TX+1]  U-part of x-face fluxes
  float *fys = fxs + 5 * TY * (TX + 1);      // [5][TY+1][TX]  U-part of y-face fluxes
  if (ctl->done) return;
  const float *w = pick(ctl, in_sel, w0, w1, wp);
  const float *wb = pick(ctl, 0, w0, w1, wp);
  float dt = dt_of(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const size_t N = (size_t)g.n;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * zc;
  const int z1 = min(z0 + zc, g.sz);
  const int x = x0 + tx, y = y0 + ty;
  const bool active = x < g.sx && y < g.sy;
  const int yw_self = wrapi(y, g.sy);
  const float gm1 = g.gamma - 1.0f;
  const bool in_place_bef = in_sel == 0;  // stage 1: W_bef is the flux input

  ZCol zw[4];
  float fz_lo[7];
  // planes z0-2 .. z1+1 enter the ring in order
  for (int pz = z0 - 2; pz <= z1 + 1; ++pz) {
    const int sl = (pz - (z0 - 2)) % 3;
    float *slot = ring + sl * SLOT;
    __syncthreads();  // everyone is done with the plane this slot held
    load_plane<TY, 2, 8, 8>(slot, w, w, g, x0, y0, pz);
    __syncthreads();
    zw[0] = zw[1];
    zw[1] = zw[2];
    zw[2] = zw[3];
    zw[3] = zcol<TY>(slot, ty, tx);
    if (pz < z0 + 1) continue;
    // z-face between planes pz-2 and pz-1 (lower face of cell plane pz-1)
    const float *slot_m1 = ring + ((pz - 1 - (z0 - 2)) % 3) * SLOT;
    float fz_hi[7];
    z_face(g, zw[0], zw[1], zw[2], zw[3], slot_m1[F_BZ * PLANE + (ty + 2) * PX + tx + 2], dt, fz_hi);
    if (pz >= z0 + 2) {
      // finalize plane k = pz - 2: x/y faces from its slot, B_z above from pz-1
      const int k = pz - 2;
      const float *sk = ring + ((k - (z0 - 2)) % 3) * SLOT;
      float fx[7], fy[7];
      xy_face<0, TY>(g, sk, slot_m1, ty, tx, yw_self, dt, fx);
      xy_face<1, TY>(g, sk, slot_m1, ty, tx, yw_self, dt, fy);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        fxs[(v * TY + ty) * (TX + 1) + tx] = fx[v];
        fys[(v * (TY + 1) + ty) * TX + tx] = fy[v];
      }
      // the faces on the far side of the tile: x-face 32 of each row (warp 1),
      // y-face TY of each column (warp 0)
      if (ty == 0) {
        float ey[7];
        xy_face<1, TY>(g, sk, slot_m1, TY, tx, wrapi(y0 + TY, g.sy), dt, ey);
#pragma unroll
        for (int v = 0; v < 5; ++v) fys[(v * (TY + 1) + TY) * TX + tx] = ey[v];
      } else if (ty == 1 && tx < TY) {
        float ex[7];
        xy_face<0, TY>(g, sk, slot_m1, tx, TX, wrapi(y0 + tx, g.sy), dt, ex);
#pragma unroll
        for (int v = 0; v < 5; ++v) fxs[(v * TY + tx) * (TX + 1) + TX] = ex[v];
      }
      __syncthreads();
      if (active && k < z1) {
        const size_t o = ((size_t)k * g.sy + y) * g.sx + x;
        // flux divergence of rho, m, E: x, then y, then z
        float pace[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          float pc = 0.0f;
          pc = pc + (fxs[(v * TY + ty) * (TX + 1) + tx] - fxs[(v * TY + ty) * (TX + 1) + tx + 1]) / g.dx;
          pc = pc + (fys[(v * (TY + 1) + ty) * TX + tx] - fys[(v * (TY + 1) + ty + 1) * TX + tx]) / g.dy;
          pc = pc + (fz_lo[v] - fz_hi[v]) / g.dz;
          pace[v] = pc;
        }
        // conserved state before the stage
        float rho0, vx0, vy0, vz0, p0, bxl, bxh, byl, byh, bzl, bzh;
        if (in_place_bef) {
          const int i = (ty + 2) * PX + tx + 2;
          rho0 = sk[F_RHO * PLANE + i];
          vx0 = sk[F_VX * PLANE + i];
          vy0 = sk[F_VY * PLANE + i];
          vz0 = sk[F_VZ * PLANE + i];
          p0 = sk[F_P * PLANE + i];
          bxl = sk[F_BX * PLANE + i];
          bxh = sk[F_BX * PLANE + i + 1];
          byl = sk[F_BY * PLANE + i];
          byh = sk[F_BY * PLANE + i + PX];
          bzl = sk[F_BZ * PLANE + i];
          bzh = slot_m1[F_BZ * PLANE + i];
        } else {
          const int xp = x + 1 < g.sx ? x + 1 : 0, yp = y + 1 < g.sy ? y + 1 : 0;
          const int kp = k + 1 < g.sz ? k + 1 : 0;
          rho0 = wb[o];
          vx0 = wb[N + o];
          vy0 = wb[2 * N + o];
          vz0 = wb[3 * N + o];
          p0 = wb[4 * N + o];
          bxl = wb[5 * N + o];
          bxh = wb[5 * N + ((size_t)k * g.sy + y) * g.sx + xp];
          byl = wb[6 * N + o];
          byh = wb[6 * N + ((size_t)k * g.sy + yp) * g.sx + x];
          bzl = wb[7 * N + o];
          bzh = wb[7 * N + ((size_t)kp * g.sy + y) * g.sx + x];
        }
        const float mx0 = rho0 * vx0, my0 = rho0 * vy0, mz0 = rho0 * vz0;
        const float e0 = p0 / gm1 + 0.5f * rho0 * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0) +
                         0.25f * (bxl * bxl + bxh * bxh + byl * byl + byh * byh + bzl * bzl + bzh * bzh);
        unew[o] = rho0 + dt * pace[0];
        unew[N + o] = mx0 + dt * pace[1];
        unew[2 * N + o] = my0 + dt * pace[2];
        unew[3 * N + o] = mz0 + dt * pace[3];
        unew[4 * N + o] = e0 + dt * pace[4];
        // B fluxes of the cell's own lower faces, for the corner EMFs
        bflux[o] = fx[5];            // F_x(B_y)
        bflux[N + o] = fx[6];        // F_x(B_z)
        bflux[2 * N + o] = fy[5];    // F_y(B_z)
        bflux[3 * N + o] = fy[6];    // F_y(B_x)
        bflux[4 * N + o] = fz_lo[5]; // F_z(B_x)
        bflux[5 * N + o] = fz_lo[6]; // F_z(B_y)
      }
    }
#pragma unroll
    for (int v = 0; v < 7; ++v) fz_lo[v] = fz_hi[v];
  }
}

// ---------------------------------------------------------------------------
// Corner (edge) flux of B_b carried by the a-flux (corner_magnet_flux,
// mhd_solver.inlrb:641-653): wind = sum of the four v_b around the edge, in the
// reference's order (e, e-b, e-a, e-a-b); upwind face e-b if positive, e if
// negative, their mean on a tie.
__device__ __forceinline__ float corner(float w_e, float w_mb, float w_ma, float w_mab, float f_mb,
                                        float f_e) {
  const float w = w_e + w_mb + w_ma + w_mab;
  return w > 0.0f ? f_mb : (w < 0.0f ? f_e : 0.5f * (f_mb + f_e));
}

// Fields of the CT ring (halo 1): B fluxes, then the flux-input velocities.
enum { G_FXBY = 0, G_FXBZ = 1, G_FYBZ = 2, G_FYBX = 3, G_FZBX = 4, G_FZBY = 5, G_VX = 6, G_VY = 7, G_VZ = 8 };

template <int TY>
struct CtView {
  static constexpr int PX = TX + 2, PLANE = PX * (TY + 2);
  const float *lo, *mid, *hi;  // planes k-1, k, k+1
  int r, c;                    // smem coordinates (+1 halo applied) of cell (i, j)
  __device__ __forceinline__ float at(const float *s, int f, int dx, int dy) const {
    return s[f * PLANE + (r + dy) * PX + (c + dx)];
  }
};

// Face-B paces (constrained transport) of the lower x-, y- and z-face of the
// cell at (r, c) of plane `mid`; the z-face uses planes lo and mid.
template <int TY>
__device__ __forceinline__ float pace_bx(const CtView<TY> &v, float dx, float dy, float dz) {
  const float *m = v.mid;
  // XY corners at edges (i, j) and (i, j+1): F_x(B_y), wind v_y
  auto XY = [&](int ey) {
    return corner(v.at(m, G_VY, 0, ey), v.at(m, G_VY, 0, ey - 1), v.at(m, G_VY, -1, ey),
                  v.at(m, G_VY, -1, ey - 1), v.at(m, G_FXBY, 0, ey - 1), v.at(m, G_FXBY, 0, ey));
  };
  // YX corners at (i, j) and (i, j+1): F_y(B_x), wind v_x
  auto YX = [&](int ey) {
    return corner(v.at(m, G_VX, 0, ey), v.at(m, G_VX, -1, ey), v.at(m, G_VX, 0, ey - 1),
                  v.at(m, G_VX, -1, ey - 1), v.at(m, G_FYBX, -1, ey), v.at(m, G_FYBX, 0, ey));
  };
  // XZ corners at (i, k) and (i, k+1): F_x(B_z), wind v_z
  auto XZ = [&](const float *s, const float *sm1) {
    return corner(v.at(s, G_VZ, 0, 0), v.at(sm1, G_VZ, 0, 0), v.at(s, G_VZ, -1, 0),
                  v.at(sm1, G_VZ, -1, 0), v.at(sm1, G_FXBZ, 0, 0), v.at(s, G_FXBZ, 0, 0));
  };
  // ZX corners at (i, k) and (i, k+1): F_z(B_x), wind v_x
  auto ZX = [&](const float *s, const float *sm1) {
    return corner(v.at(s, G_VX, 0, 0), v.at(s, G_VX, -1, 0), v.at(sm1, G_VX, 0, 0),
                  v.at(sm1, G_VX, -1, 0), v.at(s, G_FZBX, -1, 0), v.at(s, G_FZBX, 0, 0));
  };
  float pb = 0.0f;
  pb = pb + 0.5f * ((XY(1) - XY(0)) / dy + (XZ(v.hi, m) - XZ(m, v.lo)) / dz);
  pb = pb - 0.5f * (YX(1) - YX(0)) / dy;
  pb = pb - 0.5f * (ZX(v.hi, m) - ZX(m, v.lo)) / dz;
  return pb;
}

template <int TY>
__device__ __forceinline__ float pace_by(const CtView<TY> &v, float dx, float dy, float dz) {
  const float *m = v.mid;
  // XY corners at (i, j) and (i+1, j)
  auto XY = [&](int ex) {
    return corner(v.at(m, G_VY, ex, 0), v.at(m, G_VY, ex, -1), v.at(m, G_VY, ex - 1, 0),
                  v.at(m, G_VY, ex - 1, -1), v.at(m, G_FXBY, ex, -1), v.at(m, G_FXBY, ex, 0));
  };
  auto YX = [&](int ex) {
    return corner(v.at(m, G_VX, ex, 0), v.at(m, G_VX, ex - 1, 0), v.at(m, G_VX, ex, -1),
                  v.at(m, G_VX, ex - 1, -1), v.at(m, G_FYBX, ex - 1, 0), v.at(m, G_FYBX, ex, 0));
  };
  // YZ corners at (j, k) and (j, k+1): F_y(B_z), wind v_z
  auto YZ = [&](const float *s, const float *sm1) {
    return corner(v.at(s, G_VZ, 0, 0), v.at(sm1, G_VZ, 0, 0), v.at(s, G_VZ, 0, -1),
                  v.at(sm1, G_VZ, 0, -1), v.at(sm1, G_FYBZ, 0, 0), v.at(s, G_FYBZ, 0, 0));
  };
  // ZY corners at (j, k) and (j, k+1): F_z(B_y), wind v_y
  auto ZY = [&](const float *s, const float *sm1) {
    return corner(v.at(s, G_VY, 0, 0), v.at(s, G_VY, 0, -1), v.at(sm1, G_VY, 0, 0),
                  v.at(sm1, G_VY, 0, -1), v.at(s, G_FZBY, 0, -1), v.at(s, G_FZBY, 0, 0));
  };
  float pb = 0.0f;
  pb = pb - 0.5f * (XY(1) - XY(0)) / dx;
  pb = pb + 0.5f * ((YZ(v.hi, m) - YZ(m, v.lo)) / dz + (YX(1) - YX(0)) / dx);
  pb = pb - 0.5f * (ZY(v.hi, m) - ZY(m, v.lo)) / dz;
  return pb;
}

// B_z pace of the z-face between planes `lo` (below) and `mid` (the cell's plane).
template <int TY>
__device__ __forceinline__ float pace_bz(const CtView<TY> &v, float dx, float dy, float dz) {
  const float *s = v.mid, *sm1 = v.lo;
  // XZ corners at (i, k) and (i+1, k)
  auto XZ = [&](int ex) {
    return corner(v.at(s, G_VZ, ex, 0), v.at(sm1, G_VZ, ex, 0), v.at(s, G_VZ, ex - 1, 0),
                  v.at(sm1, G_VZ, ex - 1, 0), v.at(sm1, G_FXBZ, ex, 0), v.at(s, G_FXBZ, ex, 0));
  };
  auto YZ = [&](int ey) {
    return corner(v.at(s, G_VZ, 0, ey), v.at(sm1, G_VZ, 0, ey), v.at(s, G_VZ, 0, ey - 1),
                  v.at(sm1, G_VZ, 0, ey - 1), v.at(sm1, G_FYBZ, 0, ey), v.at(s, G_FYBZ, 0, ey));
  };
  auto ZX = [&](int ex) {
    return corner(v.at(s, G_VX, ex, 0), v.at(s, G_VX, ex - 1, 0), v.at(sm1, G_VX, ex, 0),
                  v.at(sm1, G_VX, ex - 1, 0), v.at(s, G_FZBX, ex - 1, 0), v.at(s, G_FZBX, ex, 0));
  };
  auto ZY = [&](int ey) {
    return corner(v.at(s, G_VY, 0, ey), v.at(s, G_VY, 0, ey - 1), v.at(sm1, G_VY, 0, ey),
                  v.at(sm1, G_VY, 0, ey - 1), v.at(s, G_FZBY, 0, ey - 1), v.at(s, G_FZBY, 0, ey));
  };
  float pb = 0.0f;
  pb = pb - 0.5f * (XZ(1) - XZ(0)) / dx;
  pb = pb - 0.5f * (YZ(1) - YZ(0)) / dy;
  pb = pb + 0.5f * ((ZX(1) - ZX(0)) / dx + (ZY(1) - ZY(0)) / dy);
  return pb;
}

__device__ __forceinline__ float block_min_2d(float v, float *red) {
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int nw = (blockDim.x * blockDim.y) >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < nw ? red[lane] : __uint_as_float(0x7f800000u);
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

template <int TY>
__global__ void __launch_bounds__(TX *TY) k_tile_ct(GridParams g, StepCtl *ctl, float *w0, float *w1,
                                                    float *wp, const float *__restrict__ unew,
                                                    const float *__restrict__ bflux, float *dt_hist,
                                                    int in_sel, int out_sel, int half, int final_stage,
                                                    int zc) {
  using V = CtView<TY>;
  constexpr int SLOT = 9 * V::PLANE;
  extern __shared__ float sm[];
  float *ring = sm;                        // [3][9][TY+2][TX+2]
  float *bxs = ring + 3 * SLOT;            // [TY][TX+1] new B_x
  float *bys = bxs + TY * (TX + 1);        // [TY+1][TX] new B_y
  __shared__ float red[32];
  __shared__ int bad_any;
  if (ctl->done) return;
  const float *win = pick(ctl, in_sel, w0, w1, wp);
  const float *wb = pick(ctl, 0, w0, w1, wp);
  float *wo = const_cast<float *>(pick(ctl, out_sel, w0, w1, wp));
  float dt = dt_of(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const size_t N = (size_t)g.n;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * zc;
  const int z1 = min(z0 + zc, g.sz);
  const int x = x0 + tx, y = y0 + ty;
  const bool active = x < g.sx && y < g.sy;
  const float gm1 = g.gamma - 1.0f;
  if (tx == 0 && ty == 0) bad_any = 0;
  float tcfl = __uint_as_float(0x7f800000u);
  int bad = 0;
  float bz_lo_new = 0.0f;
  // planes z0-1 .. z1 enter the ring; plane k = pz-1 is finalized
  for (int pz = z0 - 1; pz <= z1; ++pz) {
    const int sl = (pz - (z0 - 1)) % 3;
    __syncthreads();
    // fields 0..5: B fluxes; 6..8: velocities (fields 1..3 of the flux input)
    load_plane<TY, 1, 9, 6>(ring + sl * SLOT, bflux, win + N, g, x0, y0, pz);
    __syncthreads();
    if (pz < z0 + 1) continue;
    const int k = pz - 1;
    V v;
    v.lo = ring + ((k - 1 - (z0 - 1)) % 3) * SLOT;
    v.mid = ring + ((k - (z0 - 1)) % 3) * SLOT;
    v.hi = ring + sl * SLOT;
    v.r = ty + 1;
    v.c = tx + 1;
    const int xw = wrapi(x, g.sx), yw = wrapi(y, g.sy);
    const int kw = wrapi(k, g.sz), kpw = wrapi(k + 1, g.sz);
    const size_t o = ((size_t)kw * g.sy + yw) * g.sx + xw;
    // new face B: own lower x- and y-faces, the z-faces below and above
    const float pbx = pace_bx<TY>(v, g.dx, g.dy, g.dz);
    const float pby = pace_by<TY>(v, g.dx, g.dy, g.dz);
    const float bxn = wb[5 * N + o] + dt * pbx;
    const float byn = wb[6 * N + o] + dt * pby;
    if (pz == z0 + 1) {
      bz_lo_new = wb[7 * N + o] + dt * pace_bz<TY>(v, g.dx, g.dy, g.dz);
    }
    V vu = v;
    vu.lo = v.mid;
    vu.mid = v.hi;
    const size_t ou = ((size_t)kpw * g.sy + yw) * g.sx + xw;
    const float bz_hi_new = wb[7 * N + ou] + dt * pace_bz<TY>(vu, g.dx, g.dy, g.dz);
    bxs[ty * (TX + 1) + tx] = bxn;
    bys[ty * TX + tx] = byn;
    // far-side faces of the tile: x-face 32 of each row, y-face TY of each column
    if (ty == 0) {
      V e = v;
      e.r = TY + 1;
      const int ye = wrapi(y0 + TY, g.sy);
      const size_t oe = ((size_t)kw * g.sy + ye) * g.sx + xw;
      bys[TY * TX + tx] = wb[6 * N + oe] + dt * pace_by<TY>(e, g.dx, g.dy, g.dz);
    } else if (ty == 1 && tx < TY) {
      V e = v;
      e.r = tx + 1;
      e.c = TX + 1;
      const int xe = wrapi(x0 + TX, g.sx), ye = wrapi(y0 + tx, g.sy);
      const size_t oe = ((size_t)kw * g.sy + ye) * g.sx + xe;
      bxs[tx * (TX + 1) + TX] = wb[5 * N + oe] + dt * pace_bx<TY>(e, g.dx, g.dy, g.dz);
    }
    __syncthreads();
    if (active && k < z1) {
      const float bx0 = bxs[ty * (TX + 1) + tx], bx1 = bxs[ty * (TX + 1) + tx + 1];
      const float by0 = bys[ty * TX + tx], by1 = bys[(ty + 1) * TX + tx];
      const float bz0 = bz_lo_new, bz1 = bz_hi_new;
      const float rho = unew[o];
      const float mx = unew[N + o], my = unew[2 * N + o], mz = unew[3 * N + o];
      const float ene = unew[4 * N + o];
      float vxo = mx / rho, vyo = my / rho, vzo = mz / rho;
      const float eint = ene - 0.5f * (mx * mx + my * my + mz * mz) / rho -
                         0.25f * (bx0 * bx0 + bx1 * bx1 + by0 * by0 + by1 * by1 + bz0 * bz0 + bz1 * bz1);
      const float po = eint * gm1;
      if (g.shear) {
        const float ax = -2.0f * g.omega * vyo;
        const float ay = 2.0f * g.omega * vxo + 2.0f * g.q * (g.omega * g.omega) * kepler_y(g, y);
        vxo = vxo + dt * ax;
        vyo = vyo + dt * ay;
        vzo = vzo + dt * 0.0f;
      }
      wo[o] = rho;
      wo[N + o] = vxo;
      wo[2 * N + o] = vyo;
      wo[3 * N + o] = vzo;
      wo[4 * N + o] = po;
      wo[5 * N + o] = bx0;
      wo[6 * N + o] = by0;
      wo[7 * N + o] = bz0;
      if (final_stage) {
        bad |= !(rho > 0.0f) || !(po > 0.0f) || !isfinite(vxo) || !isfinite(vyo) || !isfinite(vzo) ||
               !isfinite(bx0) || !isfinite(by0) || !isfinite(bz0);
        const bool margin_cell = (y < g.my) || (y >= g.sy - g.my) ||
                                 (g.mz > 0 && (k < g.mz || k >= g.sz - g.mz - 1));
        if (!margin_cell) {
          const float b2 = fmaxf(bx0 * bx0, bx1 * bx1) + fmaxf(by0 * by0, by1 * by1) +
                           fmaxf(bz0 * bz0, bz1 * bz1);
          const float c = sqrtf((g.gamma * po + b2) / rho);
          const float t = fminf(fminf(g.cfl * g.dx / fabsf(vxo + c), g.cfl * g.dy / fabsf(vyo + c)),
                                g.cfl * g.dz / fabsf(vzo + c));
          tcfl = fminf(tcfl, t);
        }
      }
    }
    bz_lo_new = bz_hi_new;
  }
  if (!final_stage) return;
  tcfl = block_min_2d(tcfl, red);
  if (bad) bad_any = 1;
  __syncthreads();
  if (tx == 0 && ty == 0) {
    atomicMin(&ctl->cfl_next, __float_as_uint(tcfl));
    if (bad_any) atomicOr(&ctl->status, kStatusNumerical);
    __threadfence();
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned prev = atomicAdd(&ctl->blocks_done, 1u);
    if (prev == nblocks - 1) {
      __threadfence();
      bool last;
      const float dts = dt_of(ctl, &last);
      volatile StepCtl *vc = ctl;
      const long long gen = vc->generation;
      dt_hist[gen % kDtHistCap] = dts;
      vc->time = vc->time + (double)dts;
      vc->generation = gen + 1;
      vc->parity = vc->parity ^ 1;
      vc->cfl_cur = atomicAdd(&ctl->cfl_next, 0u);
      vc->cfl_next = 0x7f800000u;
      if (!(dts >= 0.0f)) atomicOr(&ctl->status, kStatusBadDt);
      if (last || vc->status) vc->done = 1;
      vc->blocks_done = 0;
    }
  }
}

template <int TY>
size_t flux_smem() {
  return sizeof(float) * (3 * 8 * (TX + 4) * (TY + 4) + 5 * TY * (TX + 1) + 5 * (TY + 1) * TX);
}
template <int TY>
size_t ct_smem() {
  return sizeof(float) * (3 * 9 * (TX + 2) * (TY + 2) + TY * (TX + 1) + (TY + 1) * TX);
}

// Opt in to more than 48 KB of dynamic shared memory (the attribute is per
// device; set it whenever a launch happens on a device not yet configured).
template <int TY>
void configure_smem() {
  static unsigned long long done_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(done_mask & (1ull << dev))) {
    cudaFuncSetAttribute(k_tile_flux<TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)flux_smem<TY>());
    cudaFuncSetAttribute(k_tile_ct<TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ct_smem<TY>());
    done_mask |= 1ull << dev;
  }
}

template <int TY>
dim3 tile_grid(const GridParams &g, int zc) {
  return dim3((g.sx + TX - 1) / TX, (g.sy + TY - 1) / TY, (g.sz + zc - 1) / zc);
}

template <int TY>
void flux_t(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew, float *bflux,
            int in_sel, int half, int zc, cudaStream_t st) {
  configure_smem<TY>();
  k_tile_flux<TY><<<tile_grid<TY>(g, zc), dim3(TX, TY), flux_smem<TY>(), st>>>(g, ctl, w0, w1, wp, unew,
                                                                               bflux, in_sel, half, zc);
}

template <int TY>
void ct_t(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew, float *bflux,
          float *dt_hist, int in_sel, int out_sel, int half, int final_stage, int zc, cudaStream_t st) {
  configure_smem<TY>();
  k_tile_ct<TY><<<tile_grid<TY>(g, zc), dim3(TX, TY), ct_smem<TY>(), st>>>(
      g, ctl, w0, w1, wp, unew, bflux, dt_hist, in_sel, out_sel, half, final_stage, zc);
}

int chunk(const GridParams &g, const TileShape &shape) { return shape.zc > 0 ? shape.zc : g.sz; }

}  // namespace

void launch_tile_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew,
                      float *bflux, int in_sel, int half, const TileShape &shape, cudaStream_t st) {
  const int zc = chunk(g, shape);
  if (shape.ty == 16) flux_t<16>(g, ctl, w0, w1, wp, unew, bflux, in_sel, half, zc, st);
  else if (shape.ty == 4) flux_t<4>(g, ctl, w0, w1, wp, unew, bflux, in_sel, half, zc, st);
  else flux_t<8>(g, ctl, w0, w1, wp, unew, bflux, in_sel, half, zc, st);
}

void launch_tile_ct(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew,
                    float *bflux, float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                    const TileShape &shape, cudaStream_t st) {
  const int zc = chunk(g, shape);
  if (shape.ty == 16) ct_t<16>(g, ctl, w0, w1, wp, unew, bflux, dt_hist, in_sel, out_sel, half, final_stage, zc, st);
  else if (shape.ty == 4) ct_t<4>(g, ctl, w0, w1, wp, unew, bflux, dt_hist, in_sel, out_sel, half, final_stage, zc, st);
  else ct_t<8>(g, ctl, w0, w1, wp, unew, bflux, dt_hist, in_sel, out_sel, half, final_stage, zc, st);
}

void launch_tile_stage(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *unew,
                       float *bflux, float *dt_hist, int in_sel, int out_sel, int half, int final_stage,
                       const TileShape &shape, cudaStream_t st) {
  launch_tile_flux(g, ctl, w0, w1, wp, unew, bflux, in_sel, half, shape, st);
  launch_tile_ct(g, ctl, w0, w1, wp, unew, bflux, dt_hist, in_sel, out_sel, half, final_stage, shape, st);
}

}  // namespace nmhd
