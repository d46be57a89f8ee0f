// Per-cell stage kernels (v3) of the B200 ideal-MHD time step, sm_100a.
//
// One thread per cell, 32 x 4 x 2 cells per CTA so that the stencil
// neighbours in x, y and z of a CTA mostly hit the SM's L1.  Every periodic
// neighbour address is the cell address plus one of nine offsets computed once
// per thread (wrap along x, y, z at -2, -1, +1), so the stencil gathers cost
// one add each.
//
//  k_cell_flux    reconstruction + HLLD on the cell's lower x-, y- and z-face
//                 (calc_flux_kernel<X,Y,Z>, src/library/mhd_solver.inlrb:562-636);
//                 21 flux values per cell (mass, momentum x/y/z, energy, two
//                 transverse B) go to scratch.
//  k_cell_update  flux divergence (add_flux_kernel :689-693), corner EMFs and
//                 face-B update (:641-714), conserved update (:762-835),
//                 primitive recovery (:779-795), the Kepler kick (:837-848),
//                 and in the final stage the CFL reduction and clock update
//                 (:496-521, 870-901, 981).
//
// Same arithmetic as the other variants (mhd_math.cuh, -fmad=false): results
// are bitwise identical.
#include "mhd_math.cuh"
#include "step.cuh"

namespace nmhd {

namespace {

constexpr int BX = 32, BY = 4, BZ = 2, kThreads = BX * BY * BZ;

__device__ __forceinline__ int wrap_any(int v, int s) {
  while (v < 0) v += s;
  while (v >= s) v -= s;
  return v;
}

// Offset (in elements of stride) from coordinate c to the periodic c + d.
__device__ __forceinline__ int woff(int c, int d, int s) { return wrap_any(c + d, s) - c; }

struct Offsets {
  int xm2, xm1, xp1, ym2, ym1, yp1, zm2, zm1, zp1;
};

__device__ __forceinline__ Offsets offsets(const GridParams &g, int x, int y, int z) {
  const int sxy = g.sx * g.sy;
  Offsets f;
  f.xm2 = woff(x, -2, g.sx);
  f.xm1 = woff(x, -1, g.sx);
  f.xp1 = woff(x, 1, g.sx);
  f.ym2 = woff(y, -2, g.sy) * g.sx;
  f.ym1 = woff(y, -1, g.sy) * g.sx;
  f.yp1 = woff(y, 1, g.sy) * g.sx;
  f.zm2 = woff(z, -2, g.sz) * sxy;
  f.zm1 = woff(z, -1, g.sz) * sxy;
  f.zp1 = woff(z, 1, g.sz) * sxy;
  return f;
}

__device__ __forceinline__ float cell_dt(const StepCtl *c, bool *last) {
  const float cmin = __uint_as_float(c->cfl_cur);
  float dt = fminf(c->goal, cmin);
  const double next_time = c->time + (double)dt;
  const bool l = next_time > (double)c->goal;
  if (l) dt = (float)((double)c->goal - c->time);
  if (last) *last = l;
  return dt;
}

__device__ __forceinline__ const float *cell_pick(const StepCtl *c, int sel, const float *w0,
                                                  const float *w1, const float *wp) {
  if (sel == 2) return wp;
  return (sel == 0) == (c->parity == 0) ? w0 : w1;
}

// Flux through the lower face of cell o along runtime axis `ax` (one HLLD
// instance serves all three axes, keeping the kernel's code small).
// sm/sp: offsets of the stencil cells -2, -1, +1 along ax; t1/t2: +1 offsets
// along the transverse axes ax+1 and ax+2 (mod 3).  The 7 results go to
// flux + (7*ax + k)*N + o with momentum in absolute components.
__device__ __forceinline__ void cell_face_rt(const GridParams &g, const float *__restrict__ w, size_t N,
                                             int o, int ax, int m2, int m1, int p1, int t1, int t2,
                                             int yidx, float dt, float *__restrict__ flux) {
  const int e1 = ax == 2 ? 0 : ax + 1, e2 = ax == 0 ? 2 : ax - 1;
  const float *rho = w, *p = w + 4 * N;
  const float *vn = w + (1 + ax) * N, *v1 = w + (1 + e1) * N, *v2 = w + (1 + e2) * N;
  const float *bn = w + (5 + ax) * N, *b1 = w + (5 + e1) * N, *b2 = w + (5 + e2) * N;
  const int s[4] = {m2, m1, 0, p1};
  float bc1[4], bc2[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int c = o + s[t];
    bc1[t] = 0.5f * (__ldg(b1 + c) + __ldg(b1 + c + t1));
    bc2[t] = 0.5f * (__ldg(b2 + c) + __ldg(b2 + c + t2));
  }
  HlldIn in;
  if (g.order2) {
    reconstruct4(__ldg(rho + o + m2), __ldg(rho + o + m1), __ldg(rho + o), __ldg(rho + o + p1), in.dl, in.dr);
    reconstruct4(__ldg(vn + o + m2), __ldg(vn + o + m1), __ldg(vn + o), __ldg(vn + o + p1), in.ul, in.ur);
    reconstruct4(__ldg(v1 + o + m2), __ldg(v1 + o + m1), __ldg(v1 + o), __ldg(v1 + o + p1), in.vl, in.vr);
    reconstruct4(__ldg(v2 + o + m2), __ldg(v2 + o + m1), __ldg(v2 + o), __ldg(v2 + o + p1), in.wl, in.wr);
    reconstruct4(__ldg(p + o + m2), __ldg(p + o + m1), __ldg(p + o), __ldg(p + o + p1), in.pl, in.pr);
    reconstruct4(bc1[0], bc1[1], bc1[2], bc1[3], in.byl, in.byr);
    reconstruct4(bc2[0], bc2[1], bc2[2], bc2[3], in.bzl, in.bzr);
  } else {
    in.dl = __ldg(rho + o + m1); in.dr = __ldg(rho + o);
    in.ul = __ldg(vn + o + m1); in.ur = __ldg(vn + o);
    in.vl = __ldg(v1 + o + m1); in.vr = __ldg(v1 + o);
    in.wl = __ldg(v2 + o + m1); in.wr = __ldg(v2 + o);
    in.pl = __ldg(p + o + m1); in.pr = __ldg(p + o);
    in.byl = bc1[1]; in.byr = bc1[2];
    in.bzl = bc2[1]; in.bzr = bc2[2];
  }
  if (g.shear) {
    float acc;
    if (ax == 0) {
      const float vY = 0.5f * (__ldg(w + 2 * N + o + m1) + __ldg(w + 2 * N + o));
      acc = -2.0f * g.omega * vY;
    } else if (ax == 1) {
      const float vX = 0.5f * (__ldg(w + N + o + m1) + __ldg(w + N + o));
      acc = 2.0f * g.omega * vX + 2.0f * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((float)yidx + 0.5f));
    } else {
      acc = 0.0f;
    }
    const float mbv = 0.5f * dt * acc;
    in.ul += mbv;
    in.ur += mbv;
  }
  float f[7];
  hlld_flux(g.gamma, __ldg(bn + o), in, f);
  float *out = flux + (size_t)(7 * ax) * N + o;
  out[0] = f[0];
  out[(1 + ax) * N] = f[1];
  out[(1 + e1) * N] = f[2];
  out[(1 + e2) * N] = f[3];
  out[4 * N] = f[4];
  out[5 * N] = f[5];
  out[6 * N] = f[6];
}

__global__ void __launch_bounds__(kThreads, 3) k_cell_flux(GridParams g, const StepCtl *ctl, const float *w0,
                                                           const float *w1, const float *wp,
                                                           float *__restrict__ flux, int in_sel, int half) {
  if (ctl->done) return;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = blockIdx.y * BY + threadIdx.y;
  const int z = blockIdx.z * BZ + threadIdx.z;
  if (x >= g.sx || y >= g.sy || z >= g.sz) return;
  const float *w = cell_pick(ctl, in_sel, w0, w1, wp);
  float dt = cell_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const size_t N = (size_t)g.n;
  const int o = (z * g.sy + y) * g.sx + x;
  const Offsets f = offsets(g, x, y, z);
#pragma unroll 1
  for (int ax = 0; ax < 3; ++ax) {
    const int m2 = ax == 0 ? f.xm2 : ax == 1 ? f.ym2 : f.zm2;
    const int m1 = ax == 0 ? f.xm1 : ax == 1 ? f.ym1 : f.zm1;
    const int p1 = ax == 0 ? f.xp1 : ax == 1 ? f.yp1 : f.zp1;
    const int t1 = ax == 0 ? f.yp1 : ax == 1 ? f.zp1 : f.xp1;
    const int t2 = ax == 0 ? f.zp1 : ax == 1 ? f.xp1 : f.yp1;
    cell_face_rt(g, w, N, o, ax, m2, m1, p1, t1, t2, y, dt, flux);
  }
}

// Shared-memory staging of the constrained-transport inputs: 6 face-B flux
// fields and the 3 flux-input velocities on the CTA's cells plus a 1-cell
// halo: (32+2) x (4+2) x (2+2) cells.
constexpr int HX = BX + 2, HY = BY + 2, HZ = BZ + 2, HPLANE = HX * HY * HZ;
enum { S_FXBY = 0, S_FXBZ, S_FYBZ, S_FYBX, S_FZBX, S_FZBY, S_VX, S_VY, S_VZ, S_NF };

// corner_magnet_flux (mhd_solver.inlrb:641-653) from the staged fields: the
// a-flux of B_b on the edge at staged cell index e (lower a- and b-face
// index of the edge); mb, ma: index offsets of -1 along b and a.
__device__ __forceinline__ float corner_s(const float *sm, int fw, int ff, int e, int mb, int ma) {
  const float *vw = sm + fw * HPLANE, *vf = sm + ff * HPLANE;
  const float w = vw[e] + vw[e + mb] + vw[e + ma] + vw[e + ma + mb];
  const float f0 = vf[e + mb];
  const float f1 = vf[e];
  return w > 0.0f ? f0 : (w < 0.0f ? f1 : 0.5f * (f0 + f1));
}

__device__ __forceinline__ float cell_block_min(float v) {
  __shared__ float red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tid = (threadIdx.z * BY + threadIdx.y) * BX + threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < kThreads / 32 ? red[lane] : __uint_as_float(0x7f800000u);
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

__global__ void __launch_bounds__(kThreads) k_cell_update(GridParams g, StepCtl *ctl, float *w0, float *w1,
                                                          float *wp, const float *__restrict__ flux,
                                                          float *dt_hist, int in_sel, int out_sel, int half,
                                                          int final_stage) {
  __shared__ float sm[S_NF * HPLANE];
  if (ctl->done) return;
  const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY, z0 = blockIdx.z * BZ;
  const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
  const bool inside = x < g.sx && y < g.sy && z < g.sz;
  const size_t N = (size_t)g.n;
  const float *win = cell_pick(ctl, in_sel, w0, w1, wp);
  const float *wb = cell_pick(ctl, 0, w0, w1, wp);
  float *wo = const_cast<float *>(cell_pick(ctl, out_sel, w0, w1, wp));
  float dt = cell_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const float *Fx = flux, *Fy = flux + 7 * N, *Fz = flux + 14 * N;
  {
    // stage rows of 34 cells: warp w takes rows w, w+8, ...; lanes cover x
    const int warp = (tz * BY + ty), lane = tx;
    const int xa = wrap_any(x0 - 1 + lane, g.sx);
    const int xb = lane < 2 ? wrap_any(x0 + 31 + lane, g.sx) : 0;
    for (int row = warp; row < S_NF * HZ * HY; row += kThreads / 32) {
      const int f = row / (HZ * HY);
      const int rem = row - f * (HZ * HY);
      const int kz = rem / HY, jy = rem - kz * HY;
      const size_t base = ((size_t)wrap_any(z0 - 1 + kz, g.sz) * g.sy + wrap_any(y0 - 1 + jy, g.sy)) * g.sx;
      // staged field f: B fluxes 5, 6 of face direction f/2, then velocities
      const float *sp = (f < 6 ? flux + (size_t)(7 * (f >> 1) + 5 + (f & 1)) * N : win + (size_t)(f - 5) * N) + base;
      float *dp = sm + f * HPLANE + (kz * HY + jy) * HX;
      dp[lane] = __ldg(sp + xa);
      if (lane < 2) dp[32 + lane] = __ldg(sp + xb);
    }
  }
  __syncthreads();
  float tcfl = __uint_as_float(0x7f800000u);
  int bad = 0;
  if (inside) {
    const int o = (z * g.sy + y) * g.sx + x;
    const Offsets f = offsets(g, x, y, z);
    const int xp = f.xp1, yp = f.yp1, zp = f.zp1;
    // flux divergence of rho, m, E (add_flux_kernel :689-693), x then y then z
    float pace[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      float pc = 0.0f;
      pc = pc + (__ldg(Fx + v * N + o) - __ldg(Fx + v * N + o + xp)) / g.dx;
      pc = pc + (__ldg(Fy + v * N + o) - __ldg(Fy + v * N + o + yp)) / g.dy;
      pc = pc + (__ldg(Fz + v * N + o) - __ldg(Fz + v * N + o + zp)) / g.dz;
      pace[v] = pc;
    }
    // corner EMFs on the 4 edges of each plane touching the cell's faces
    const int c = ((tz + 1) * HY + (ty + 1)) * HX + (tx + 1);
    const int DX = 1, DY = HX, DZ = HX * HY;
    float XY[2][2], YX[2][2], XZ[2][2], ZX[2][2], YZ[2][2], ZY[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        // XY: F_x(B_y), wind v_y, edge (x+i, y+j); mb = -y, ma = -x
        XY[i][j] = corner_s(sm, S_VY, S_FXBY, c + i * DX + j * DY, -DY, -DX);
        // YX: F_y(B_x), wind v_x; mb = -x, ma = -y
        YX[i][j] = corner_s(sm, S_VX, S_FYBX, c + i * DX + j * DY, -DX, -DY);
        // XZ: F_x(B_z), wind v_z, edge (x+i, z+j); mb = -z, ma = -x
        XZ[i][j] = corner_s(sm, S_VZ, S_FXBZ, c + i * DX + j * DZ, -DZ, -DX);
        // ZX: F_z(B_x), wind v_x; mb = -x, ma = -z
        ZX[i][j] = corner_s(sm, S_VX, S_FZBX, c + i * DX + j * DZ, -DX, -DZ);
        // YZ: F_y(B_z), wind v_z, edge (y+i, z+j); mb = -z, ma = -y
        YZ[i][j] = corner_s(sm, S_VZ, S_FYBZ, c + i * DY + j * DZ, -DZ, -DY);
        // ZY: F_z(B_y), wind v_y; mb = -y, ma = -z
        ZY[i][j] = corner_s(sm, S_VY, S_FZBY, c + i * DY + j * DZ, -DY, -DZ);
      }
    }
    float pbx[2], pby[2], pbz[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      float pb = 0.0f;
      pb = pb + 0.5f * ((XY[k][1] - XY[k][0]) / g.dy + (XZ[k][1] - XZ[k][0]) / g.dz);
      pb = pb - 0.5f * (YX[k][1] - YX[k][0]) / g.dy;
      pb = pb - 0.5f * (ZX[k][1] - ZX[k][0]) / g.dz;
      pbx[k] = pb;
      pb = 0.0f;
      pb = pb - 0.5f * (XY[1][k] - XY[0][k]) / g.dx;
      pb = pb + 0.5f * ((YZ[k][1] - YZ[k][0]) / g.dz + (YX[1][k] - YX[0][k]) / g.dx);
      pb = pb - 0.5f * (ZY[k][1] - ZY[k][0]) / g.dz;
      pby[k] = pb;
      pb = 0.0f;
      pb = pb - 0.5f * (XZ[1][k] - XZ[0][k]) / g.dx;
      pb = pb - 0.5f * (YZ[1][k] - YZ[0][k]) / g.dy;
      pb = pb + 0.5f * ((ZX[1][k] - ZX[0][k]) / g.dx + (ZY[1][k] - ZY[0][k]) / g.dy);
      pbz[k] = pb;
    }
    // conserved state before the stage (to_conserved_kernel :762-777), update
    // (add_pace/update :797-835), primitive recovery (:779-795)
    const float gm1 = g.gamma - 1.0f;
    const float rho0 = wb[o];
    const float vx0 = wb[N + o], vy0 = wb[2 * N + o], vz0 = wb[3 * N + o], p0 = wb[4 * N + o];
    float bx[2] = {wb[5 * N + o], wb[5 * N + o + xp]};
    float by[2] = {wb[6 * N + o], wb[6 * N + o + yp]};
    float bz[2] = {wb[7 * N + o], wb[7 * N + o + zp]};
    const float mx0 = rho0 * vx0, my0 = rho0 * vy0, mz0 = rho0 * vz0;
    const float e0 = p0 / gm1 + 0.5f * rho0 * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0) +
                     0.25f * (bx[0] * bx[0] + bx[1] * bx[1] + by[0] * by[0] + by[1] * by[1] +
                              bz[0] * bz[0] + bz[1] * bz[1]);
    const float rho = rho0 + dt * pace[0];
    const float mx = mx0 + dt * pace[1];
    const float my = my0 + dt * pace[2];
    const float mz = mz0 + dt * pace[3];
    const float ene = e0 + dt * pace[4];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      bx[k] = bx[k] + dt * pbx[k];
      by[k] = by[k] + dt * pby[k];
      bz[k] = bz[k] + dt * pbz[k];
    }
    float vxo = mx / rho, vyo = my / rho, vzo = mz / rho;
    const float eint = ene - 0.5f * (mx * mx + my * my + mz * mz) / rho -
                       0.25f * (bx[0] * bx[0] + bx[1] * bx[1] + by[0] * by[0] + by[1] * by[1] +
                                bz[0] * bz[0] + bz[1] * bz[1]);
    const float po = eint * gm1;
    if (g.shear) {
      // external_acceleration_kernel (:837-848) with the Kepler hook
      const float ax = -2.0f * g.omega * vyo;
      const float ay = 2.0f * g.omega * vxo + 2.0f * g.q * (g.omega * g.omega) * (g.corner_y + g.dy * ((float)y + 0.5f));
      vxo = vxo + dt * ax;
      vyo = vyo + dt * ay;
      vzo = vzo + dt * 0.0f;
    }
    wo[o] = rho;
    wo[N + o] = vxo;
    wo[2 * N + o] = vyo;
    wo[3 * N + o] = vzo;
    wo[4 * N + o] = po;
    wo[5 * N + o] = bx[0];
    wo[6 * N + o] = by[0];
    wo[7 * N + o] = bz[0];
    if (final_stage) {
      bad = !(rho > 0.0f) || !(po > 0.0f) || !isfinite(vxo) || !isfinite(vyo) || !isfinite(vzo) ||
            !isfinite(bx[0]) || !isfinite(by[0]) || !isfinite(bz[0]);
      const bool margin_cell = (y < g.my) || (y >= g.sy - g.my) ||
                               (g.mz > 0 && (z < g.mz || z >= g.sz - g.mz - 1));
      if (!margin_cell) {
        const float b2 = fmaxf(bx[0] * bx[0], bx[1] * bx[1]) + fmaxf(by[0] * by[0], by[1] * by[1]) +
                         fmaxf(bz[0] * bz[0], bz[1] * bz[1]);
        const float cs = sqrtf((g.gamma * po + b2) / rho);
        tcfl = fminf(fminf(g.cfl * g.dx / fabsf(vxo + cs), g.cfl * g.dy / fabsf(vyo + cs)),
                     g.cfl * g.dz / fabsf(vzo + cs));
      }
    }
  }
  if (!final_stage) return;
  tcfl = cell_block_min(tcfl);
  bad = __syncthreads_or(bad);
  if (tx == 0 && ty == 0 && tz == 0) {
    atomicMin(&ctl->cfl_next, __float_as_uint(tcfl));
    if (bad) atomicOr(&ctl->status, kStatusNumerical);
    __threadfence();
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned prev = atomicAdd(&ctl->blocks_done, 1u);
    if (prev == nblocks - 1) {
      // last block: advance the clock (GlobalSetup::proceed, :981) and rotate
      __threadfence();
      bool last;
      const float dts = cell_dt(ctl, &last);
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

dim3 cell_grid(const GridParams &g) {
  return dim3((g.sx + BX - 1) / BX, (g.sy + BY - 1) / BY, (g.sz + BZ - 1) / BZ);
}

}  // namespace

void launch_cell_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                      int in_sel, int half, cudaStream_t st) {
  k_cell_flux<<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, half);
}

void launch_cell_update(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                        float *dt_hist, int in_sel, int out_sel, int half, int final_stage, cudaStream_t st) {
  k_cell_update<<<cell_grid(g), dim3(BX, BY, BZ), 0, st>>>(g, ctl, w0, w1, wp, flux, dt_hist, in_sel,
                                                           out_sel, half, final_stage);
}

}  // namespace nmhd
