// Step kernels of the B200-native ideal-MHD solver (sm_100a).
//
// The reference (src/library/mhd_solver.inlrb) runs ~24 grid-stride kernels
// per RK2 step with pace/flux arrays in global memory and a blocking Thrust
// reduction for dt.  Here one RK stage is two kernels:
//   k_flux   - reconstruction + HLLD on the three lower faces of every cell
//              (calc_flux_kernel<X,Y,Z>, mhd_solver.inlrb:562-636);
//   k_update - flux divergence, constrained-transport corner EMFs, conserved
//              update, primitive recovery and the source kick of one cell
//              (add_flux_kernel, to_conserved, add_pace/update, to_primitive,
//              external_acceleration: mhd_solver.inlrb:668-848), plus, in the
//              final stage, the CFL reduction for the next step and the clock
//              update (mhd_solver.inlrb:496-521, 870-901, 981).
// The shearing-periodic margin fill (communicate(), mhd_solver.inlrb:184-493 on
// one rank) is one kernel with no buffers or host staging.
//
// All arithmetic follows the reference operation by operation (mhd_math.cuh);
// this file is compiled with -fmad=false.
#include "margin_ops.cuh"
#include "mhd_math.cuh"
#include "step.cuh"

namespace nmhd {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ int wrapc(int v, int s) {
  while (v < 0) v += s;
  while (v >= s) v -= s;
  return v;
}

struct Cell {
  int x, y, z;
};

__device__ __forceinline__ int at(const GridParams &g, int x, int y, int z) {
  return (wrapc(z, g.sz) * g.sy + wrapc(y, g.sy)) * g.sx + wrapc(x, g.sx);
}

__device__ __forceinline__ Cell decompose(const GridParams &g, int idx) {
  Cell c;
  c.x = idx % g.sx;
  int t = idx / g.sx;
  c.y = t % g.sy;
  c.z = t / g.sy;
  return c;
}

// Time step of the current step: min(goal, CFL) clamped to the goal
// (mhd_solver.inlrb:870-901).
__device__ __forceinline__ float step_dt(const StepCtl *c, bool *last) {
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

__device__ __forceinline__ const float *sel_buf(const StepCtl *c, int sel, const float *w0,
                                                const float *w1, const float *wp) {
  if (sel == 2) return wp;
  const int cur = c->parity;
  return (sel == 0) == (cur == 0) ? w0 : w1;
}

// Kepler radial coordinate of index y: RCo::position adds half a cell for
// every staggering (src/library/crystal.hrb:55-62).
__device__ __forceinline__ float kepler_y(const GridParams &g, int y) {
  return g.corner_y + g.dy * ((float)y + 0.5f);
}

// CFL time of one cell (cfl_condition_inner/kernel, mhd_solver.inlrb:496-521)
// from its primitive state and the squares of its face fields.
__device__ __forceinline__ float cfl_time(const GridParams &g, float rho, float vx, float vy,
                                          float vz, float p, float b2) {
  const float c = sqrtf((g.gamma * p + b2) / rho);
  const float tx = g.cfl * g.dx / fabsf(vx + c);
  const float ty = g.cfl * g.dy / fabsf(vy + c);
  const float tz = g.cfl * g.dz / fabsf(vz + c);
  return fminf(fminf(tx, ty), tz);
}

__device__ __forceinline__ float block_min(float v) {
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : __uint_as_float(0x7f800000u);
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

__device__ __forceinline__ float cell_cfl(const GridParams &g, const float *w, int x, int y, int z) {
  return margin::cfl_of_cell(g, w, x, y, z);
}

// ---------------------------------------------------------------------------
// CFL over all cells (first step after a state change) or over the margin set
// (every step when margins exist; interior cells are reduced by the final
// stage of the previous step, which the margin fill does not change).
__global__ void __launch_bounds__(kBlock) k_cfl(GridParams g, StepCtl *ctl, const float *w0,
                                                const float *w1, int margin_only) {
  if (ctl->done) return;
  const float *w = ctl->parity ? w1 : w0;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  float t = __uint_as_float(0x7f800000u);
  if (!margin_only) {
    if (idx < g.n) {
      const Cell c = decompose(g, idx);
      t = cell_cfl(g, w, c.x, c.y, c.z);
    }
  } else {
    if (idx < margin::margin_cfl_cells(g)) {
      int x, y, z;
      margin::margin_cfl_cell(g, idx, &x, &y, &z);
      t = cell_cfl(g, w, x, y, z);
    }
  }
  t = block_min(t);
  if (threadIdx.x == 0) atomicMin(&ctl->cfl_cur, __float_as_uint(t));
}

// ---------------------------------------------------------------------------
// Shearing-periodic Y-margin fill (communicate_gather/scatter_kernel_y,
// mhd_solver.inlrb:184-242, with relative_displacement :244-259) for one rank:
// bottom margin row j <- top interior row Sy-2M+j shifted by +d_int in x,
// vx - relative_velocity; top margin row Sy-M+j <- bottom interior row M+j
// shifted by -d_int-1, vx + relative_velocity; By of row Sy-M is kept.  The
// reference's two-point interpolation weights both multiply the same sample;
// that arithmetic is kept.
__global__ void __launch_bounds__(kBlock) k_fill_y(GridParams g, StepCtl *ctl, float *w0, float *w1) {
  if (ctl->done) return;
  float *w = ctl->parity ? w1 : w0;
  const int M = g.my;
  const int total = g.sx * M * g.sz;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  margin::fill_y_item(g, ctl->time, w, idx);
}

// Margin fill of the RK2 predictor wp before the second stage
// (NMHD_FLAG_HALO_PER_STAGE): Y shear fill at the predictor's time t + dt/2,
// then (second launch) the Z copy.
__global__ void __launch_bounds__(kBlock) k_fill_predictor_y(GridParams g, StepCtl *ctl, float *wp) {
  if (ctl->done) return;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.sx * g.my * g.sz) return;
  float dt = step_dt(ctl, nullptr);
  dt = dt / 2.0f;
  margin::fill_y_item(g, ctl->time + (double)dt, wp, idx);
}

__global__ void __launch_bounds__(kBlock) k_fill_predictor_z(GridParams g, StepCtl *ctl, float *wp) {
  if (ctl->done) return;
  const int unit = g.sx * g.sy * g.mz;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= unit) return;
  const int n = g.n;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    float *var = wp + v * n;
    const float lo = var[n - 2 * unit + idx];
    const float hi = var[unit + idx];
    var[idx] = lo;
    var[n - unit + idx] = hi;
  }
}

// Halo exchange of a radial slab (kParallelSizeY > 1), split around the
// caller's transport: k_halo_pack gathers this slab's shear-shifted boundary
// rows into the two outgoing messages, k_halo_unpack scatters the two
// incoming messages into the Y margins.  Message layout (the reference's
// mpi_buffer_y_*): field v of item (sz*M + sy)*Sx + sx at v*Sx*M*Sz + item.
__global__ void __launch_bounds__(kBlock) k_halo_pack(GridParams g, StepCtl *ctl, const float *w0,
                                                      const float *w1, float *send_inc, float *send_dec) {
  if (ctl->done) return;
  const float *w = ctl->parity ? w1 : w0;
  const int unit = g.sx * g.my * g.sz;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= unit) return;
  float inc[8], dec[8];
  margin::gather_y_item(g, margin::shear_shift(g, ctl->time), w, idx, inc, dec);
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    send_inc[(size_t)v * unit + idx] = inc[v];
    send_dec[(size_t)v * unit + idx] = dec[v];
  }
}

__global__ void __launch_bounds__(kBlock) k_halo_unpack(GridParams g, StepCtl *ctl, float *w0, float *w1,
                                                        const float *recv_inc, const float *recv_dec) {
  if (ctl->done) return;
  float *w = ctl->parity ? w1 : w0;
  const int unit = g.sx * g.my * g.sz;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= unit) return;
  float inc[8], dec[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    inc[v] = recv_inc[(size_t)v * unit + idx];
    dec[v] = recv_dec[(size_t)v * unit + idx];
  }
  margin::scatter_y_item(g, w, idx, inc, dec);
}

// Minimum of the CFL times of n slabs of one process (the MPI_Allreduce MIN of
// proceed(), mhd_solver.inlrb:870-893), written back to every slab.
__global__ void k_cfl_min(CflSlots slots) {
  if (threadIdx.x != 0) return;
  float m = *slots.p[0];
  for (int i = 1; i < slots.n; ++i) m = fminf(m, *slots.p[i]);
  for (int i = 0; i < slots.n; ++i) *slots.p[i] = m;
}

// Plain periodic Z-margin copy (the Z part of communicate(), mhd_solver.inlrb:384-402, 463-480).
__global__ void __launch_bounds__(kBlock) k_fill_z(GridParams g, StepCtl *ctl, float *w0, float *w1) {
  if (ctl->done) return;
  float *w = ctl->parity ? w1 : w0;
  const int unit = g.sx * g.sy * g.mz;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= unit) return;
  const int n = g.n;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    float *var = w + v * n;
    const float lo = var[n - 2 * unit + idx];
    const float hi = var[unit + idx];
    var[idx] = lo;
    var[n - unit + idx] = hi;
  }
}

// ---------------------------------------------------------------------------
// Flux through the lower AX-face of cell c (calc_flux_kernel<EX>).
// out: mass, momentum x/y/z (absolute components), energy, F(B_ey), F(B_ez)
// with (ey, ez) = (AX+1, AX+2) mod 3.
template <int AX>
__device__ __forceinline__ void face_flux(const GridParams &g, const float *__restrict__ w, int x,
                                          int y, int z, float dt, float out[7]) {
  constexpr int EY = (AX + 1) % 3, EZ = (AX + 2) % 3;
  const int n = g.n;
  int a[4], ay[4], az[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    int c[3] = {x, y, z};
    c[AX] += t - 2;
    a[t] = at(g, c[0], c[1], c[2]);
    int cy[3] = {c[0], c[1], c[2]};
    cy[EY] += 1;
    ay[t] = at(g, cy[0], cy[1], cy[2]);
    int cz[3] = {c[0], c[1], c[2]};
    cz[EZ] += 1;
    az[t] = at(g, cz[0], cz[1], cz[2]);
  }
  const float *rho = w, *p = w + 4 * n;
  const float *vex = w + (1 + AX) * n, *vey = w + (1 + EY) * n, *vez = w + (1 + EZ) * n;
  const float *bex = w + (5 + AX) * n, *bey = w + (5 + EY) * n, *bez = w + (5 + EZ) * n;
  HlldIn s;
  float byc[4], bzc[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    byc[t] = 0.5f * (__ldg(bey + a[t]) + __ldg(bey + ay[t]));
    bzc[t] = 0.5f * (__ldg(bez + a[t]) + __ldg(bez + az[t]));
  }
  if (g.order2) {
    reconstruct4(__ldg(rho + a[0]), __ldg(rho + a[1]), __ldg(rho + a[2]), __ldg(rho + a[3]), s.dl, s.dr);
    reconstruct4(__ldg(vex + a[0]), __ldg(vex + a[1]), __ldg(vex + a[2]), __ldg(vex + a[3]), s.ul, s.ur);
    reconstruct4(__ldg(vey + a[0]), __ldg(vey + a[1]), __ldg(vey + a[2]), __ldg(vey + a[3]), s.vl, s.vr);
    reconstruct4(__ldg(vez + a[0]), __ldg(vez + a[1]), __ldg(vez + a[2]), __ldg(vez + a[3]), s.wl, s.wr);
    reconstruct4(__ldg(p + a[0]), __ldg(p + a[1]), __ldg(p + a[2]), __ldg(p + a[3]), s.pl, s.pr);
    reconstruct4(byc[0], byc[1], byc[2], byc[3], s.byl, s.byr);
    reconstruct4(bzc[0], bzc[1], bzc[2], bzc[3], s.bzl, s.bzr);
  } else {
    s.dl = __ldg(rho + a[1]); s.dr = __ldg(rho + a[2]);
    s.ul = __ldg(vex + a[1]); s.ur = __ldg(vex + a[2]);
    s.vl = __ldg(vey + a[1]); s.vr = __ldg(vey + a[2]);
    s.wl = __ldg(vez + a[1]); s.wr = __ldg(vez + a[2]);
    s.pl = __ldg(p + a[1]); s.pr = __ldg(p + a[2]);
    s.byl = byc[1]; s.byr = byc[2];
    s.bzl = bzc[1]; s.bzr = bzc[2];
  }
  if (g.shear) {
    // face-centred Kepler acceleration: velocities averaged across the face
    float acc;
    if (AX == 0) {
      const float vY = 0.5f * (__ldg(w + 2 * n + a[1]) + __ldg(w + 2 * n + a[2]));
      acc = -2.0f * g.omega * vY;
    } else if (AX == 1) {
      const float vX = 0.5f * (__ldg(w + n + a[1]) + __ldg(w + n + a[2]));
      acc = 2.0f * g.omega * vX + 2.0f * g.q * (g.omega * g.omega) * kepler_y(g, y);
    } else {
      acc = 0.0f;
    }
    const float mbv = 0.5f * dt * acc;
    s.ul += mbv;
    s.ur += mbv;
  }
  float f[7];
  hlld_flux(g.gamma, __ldg(bex + a[2]), s, f);
  out[0] = f[0];
  out[1 + AX] = f[1];
  out[1 + EY] = f[2];
  out[1 + EZ] = f[3];
  out[4] = f[4];
  out[5] = f[5];
  out[6] = f[6];
}

__global__ void __launch_bounds__(kBlock) k_flux(GridParams g, const StepCtl *ctl, const float *w0,
                                                 const float *w1, const float *wp,
                                                 float *__restrict__ flux, int in_sel, int half) {
  if (ctl->done) return;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.n) return;
  const float *w = sel_buf(ctl, in_sel, w0, w1, wp);
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  const Cell c = decompose(g, idx);
  const int n = g.n;
  float out[7];
  const size_t N = (size_t)n;
  face_flux<0>(g, w, c.x, c.y, c.z, dt, out);
#pragma unroll
  for (int v = 0; v < 7; ++v) flux[v * N + idx] = out[v];
  face_flux<1>(g, w, c.x, c.y, c.z, dt, out);
#pragma unroll
  for (int v = 0; v < 7; ++v) flux[(7 + v) * N + idx] = out[v];
  face_flux<2>(g, w, c.x, c.y, c.z, dt, out);
#pragma unroll
  for (int v = 0; v < 7; ++v) flux[(14 + v) * N + idx] = out[v];
}

// ---------------------------------------------------------------------------
// Corner (edge) flux of B_b carried by the a-flux (corner_magnet_flux,
// mhd_solver.inlrb:641-653): upwind by the sign of the sum of the four cell
// velocities v_b around the edge; mean on a tie.  `e` is the edge with lower
// a- and b-face index e; `ea`, `eb` are address offsets of -1 along a and b.
__device__ __forceinline__ float corner_flux(const float *__restrict__ vb, const float *__restrict__ fb,
                                             int e, int e_mb, int e_ma, int e_mab) {
  const float w = __ldg(vb + e) + __ldg(vb + e_mb) + __ldg(vb + e_ma) + __ldg(vb + e_mab);
  const float f0 = __ldg(fb + e_mb);
  const float f1 = __ldg(fb + e);
  return w > 0.0f ? f0 : (w < 0.0f ? f1 : 0.5f * (f0 + f1));
}

__global__ void __launch_bounds__(kBlock) k_update(GridParams g, StepCtl *ctl, float *w0, float *w1,
                                                   float *wp, const float *__restrict__ flux,
                                                   float *dt_hist, int in_sel, int out_sel, int half,
                                                   int final_stage) {
  if (ctl->done) return;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = g.n;
  const float *win = sel_buf(ctl, in_sel, w0, w1, wp);
  const float *wb = sel_buf(ctl, 0, w0, w1, wp);
  float *wo = const_cast<float *>(sel_buf(ctl, out_sel, w0, w1, wp));
  float dt = step_dt(ctl, nullptr);
  if (half) dt = dt / 2.0f;
  float tcfl = __uint_as_float(0x7f800000u);
  int bad = 0;
  if (idx < n) {
    const Cell c = decompose(g, idx);
    const int x = c.x, y = c.y, z = c.z;
    // wrapped neighbour addresses in the 3x3x3 block around the cell
    const int xm = wrapc(x - 1, g.sx), xp = wrapc(x + 1, g.sx);
    const int ym = wrapc(y - 1, g.sy), yp = wrapc(y + 1, g.sy);
    const int zm = wrapc(z - 1, g.sz), zp = wrapc(z + 1, g.sz);
    auto A = [&](int xx, int yy, int zz) { return (zz * g.sy + yy) * g.sx + xx; };
    const int o = idx;
    const int oxp = A(xp, y, z), oyp = A(x, yp, z), ozp = A(x, y, zp);
    const size_t N = (size_t)n;
    const float *Fx = flux, *Fy = flux + 7 * N, *Fz = flux + 14 * N;

    // flux divergence of rho, m, E (add_flux_kernel, :689-693), x then y then z
    float pace[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      float pc = 0.0f;
      pc = pc + (__ldg(Fx + v * N + o) - __ldg(Fx + v * N + oxp)) / g.dx;
      pc = pc + (__ldg(Fy + v * N + o) - __ldg(Fy + v * N + oyp)) / g.dy;
      pc = pc + (__ldg(Fz + v * N + o) - __ldg(Fz + v * N + ozp)) / g.dz;
      pace[v] = pc;
    }

    // constrained transport: corner fluxes on the 4 edges of each plane that
    // touch the cell's six faces (:641-714)
    const float *vx = win + n, *vy = win + 2 * n, *vz = win + 3 * n;
    const float *FxBy = Fx + 5 * N, *FxBz = Fx + 6 * N;
    const float *FyBz = Fy + 5 * N, *FyBx = Fy + 6 * N;
    const float *FzBx = Fz + 5 * N, *FzBy = Fz + 6 * N;
    // xy-plane edges (ix, iy) in {x, x+1} x {y, y+1}
    float XY[2][2], YX[2][2], XZ[2][2], ZX[2][2], YZ[2][2], ZY[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int ex = i ? xp : x, exm = i ? x : xm;
        const int ey = j ? yp : y, eym = j ? y : ym;
        // XY: F_x(B_y), wind v_y; YX: F_y(B_x), wind v_x
        XY[i][j] = corner_flux(vy, FxBy, A(ex, ey, z), A(ex, eym, z), A(exm, ey, z), A(exm, eym, z));
        YX[i][j] = corner_flux(vx, FyBx, A(ex, ey, z), A(exm, ey, z), A(ex, eym, z), A(exm, eym, z));
        const int ez = j ? zp : z, ezm = j ? z : zm;
        // XZ: F_x(B_z), wind v_z; ZX: F_z(B_x), wind v_x  (plane index (i: x, j: z))
        XZ[i][j] = corner_flux(vz, FxBz, A(ex, y, ez), A(ex, y, ezm), A(exm, y, ez), A(exm, y, ezm));
        ZX[i][j] = corner_flux(vx, FzBx, A(ex, y, ez), A(exm, y, ez), A(ex, y, ezm), A(exm, y, ezm));
        const int fy = i ? yp : y, fym = i ? y : ym;
        // YZ: F_y(B_z), wind v_z; ZY: F_z(B_y), wind v_y  (plane index (i: y, j: z))
        YZ[i][j] = corner_flux(vz, FyBz, A(x, fy, ez), A(x, fy, ezm), A(x, fym, ez), A(x, fym, ezm));
        ZY[i][j] = corner_flux(vy, FzBy, A(x, fy, ez), A(x, fym, ez), A(x, fy, ezm), A(x, fym, ezm));
      }
    }
    // pace of B on the lower (k=0) and upper (k=1) face of each direction
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

    // conserved state before the stage (to_conserved_kernel, :762-777)
    const float gm1 = g.gamma - 1.0f;
    const float rho0 = wb[o];
    const float vx0 = wb[n + o], vy0 = wb[2 * n + o], vz0 = wb[3 * n + o], p0 = wb[4 * n + o];
    float bx[2] = {wb[5 * n + o], wb[5 * n + oxp]};
    float by[2] = {wb[6 * n + o], wb[6 * n + oyp]};
    float bz[2] = {wb[7 * n + o], wb[7 * n + ozp]};
    const float mx0 = rho0 * vx0, my0 = rho0 * vy0, mz0 = rho0 * vz0;
    const float e0 = p0 / gm1 + 0.5f * rho0 * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0) +
                     0.25f * (bx[0] * bx[0] + bx[1] * bx[1] + by[0] * by[0] + by[1] * by[1] +
                              bz[0] * bz[0] + bz[1] * bz[1]);
    // update (add_pace_kernel / update_kernel, :797-835)
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
    // primitive recovery (to_primitive_kernel, :779-795)
    float vxo = mx / rho, vyo = my / rho, vzo = mz / rho;
    const float eint = ene - 0.5f * (mx * mx + my * my + mz * mz) / rho -
                       0.25f * (bx[0] * bx[0] + bx[1] * bx[1] + by[0] * by[0] + by[1] * by[1] +
                                bz[0] * bz[0] + bz[1] * bz[1]);
    const float po = eint * gm1;
    // source kick (external_acceleration_kernel, :837-848; Kepler hook)
    if (g.shear) {
      const float ax = -2.0f * g.omega * vyo;
      const float ay = 2.0f * g.omega * vxo + 2.0f * g.q * (g.omega * g.omega) * kepler_y(g, y);
      vxo = vxo + dt * ax;
      vyo = vyo + dt * ay;
      vzo = vzo + dt * 0.0f;
    }
    wo[o] = rho;
    wo[n + o] = vxo;
    wo[2 * n + o] = vyo;
    wo[3 * n + o] = vzo;
    wo[4 * n + o] = po;
    wo[5 * n + o] = bx[0];
    wo[6 * n + o] = by[0];
    wo[7 * n + o] = bz[0];
    if (final_stage) {
      bad = !(rho > 0.0f) || !(po > 0.0f) || !isfinite(vxo) || !isfinite(vyo) || !isfinite(vzo) ||
            !isfinite(bx[0]) || !isfinite(by[0]) || !isfinite(bz[0]);
      const bool margin_cell = (y < g.my) || (y >= g.sy - g.my) ||
                               (g.mz > 0 && (z < g.mz || z >= g.sz - g.mz - 1));
      if (!margin_cell) {
        const float b2 = fmaxf(bx[0] * bx[0], bx[1] * bx[1]) + fmaxf(by[0] * by[0], by[1] * by[1]) +
                         fmaxf(bz[0] * bz[0], bz[1] * bz[1]);
        tcfl = cfl_time(g, rho, vxo, vyo, vzo, po, b2);
      }
    }
  }
  if (!final_stage) return;
  tcfl = block_min(tcfl);
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) {
    atomicMin(&ctl->cfl_next, __float_as_uint(tcfl));
    if (bad) atomicOr(&ctl->status, kStatusNumerical);
    __threadfence();
    const unsigned prev = atomicAdd(&ctl->blocks_done, 1u);
    if (prev == gridDim.x - 1) {
      // last block: advance the clock (GlobalSetup::proceed, :981) and rotate
      __threadfence();
      bool last;
      const float dts = step_dt(ctl, &last);
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

// ---------------------------------------------------------------------------
// FP64 diagnostics of the current state over the interior (and <B^2> over all
// faces, as the Kepler monitor does).
__global__ void __launch_bounds__(kBlock) k_diag(GridParams g, const StepCtl *ctl, const float *w0,
                                                 const float *w1, double *acc) {
  const float *w = ctl->parity ? w1 : w0;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = g.n;
  double v[kDiagFields];
#pragma unroll
  for (int i = 0; i < kDiagFields; ++i) v[i] = 0.0;
  double divb = 0.0;
  if (idx < n) {
    const Cell c = decompose(g, idx);
    const double bxl = w[5 * n + idx], byl = w[6 * n + idx];
    v[9] = bxl * bxl;   // <Bx^2> numerator over all faces
    v[10] = byl * byl;  // <By^2>
    const bool inner = c.y >= g.my && c.y < g.sy - g.my && c.z >= g.mz && c.z < g.sz - g.mz;
    if (inner) {
      const double dv = (double)g.dx * (double)g.dy * (double)g.dz;
      const double rho = w[idx], ux = w[n + idx], uy = w[2 * n + idx], uz = w[3 * n + idx];
      const double p = w[4 * n + idx];
      const double bxh = w[5 * n + at(g, c.x + 1, c.y, c.z)];
      const double byh = w[6 * n + at(g, c.x, c.y + 1, c.z)];
      const double bzl = w[7 * n + idx], bzh = w[7 * n + at(g, c.x, c.y, c.z + 1)];
      v[0] = rho * dv;
      v[1] = rho * ux * dv;
      v[2] = rho * uy * dv;
      v[3] = rho * uz * dv;
      v[4] = 0.5 * rho * (ux * ux + uy * uy + uz * uz) * dv;
      v[5] = p / ((double)g.gamma - 1.0) * dv;
      v[6] = 0.25 * (bxl * bxl + bxh * bxh + byl * byl + byh * byh + bzl * bzl + bzh * bzh) * dv;
      v[7] = -(0.25 * (bxl + bxh) * (byl + byh)) * dv;  // -Bx By at the cell centre
      v[8] = dv;
      divb = fabs((bxh - bxl) / (double)g.dx + (byh - byl) / (double)g.dy + (bzh - bzl) / (double)g.dz);
    }
  }
  __shared__ double red[kDiagFields][kBlock / 32];
  __shared__ double redmax[kBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < kDiagFields; ++i) {
    double s = v[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[i][warp] = s;
  }
  for (int o = 16; o > 0; o >>= 1) divb = fmax(divb, __shfl_xor_sync(0xffffffffu, divb, o));
  if (lane == 0) redmax[warp] = divb;
  __syncthreads();
  if (threadIdx.x < kDiagFields - 1) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[threadIdx.x][k];
    atomicAdd(acc + threadIdx.x, s);
  }
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmax(m, redmax[k]);
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(acc + kDiagFields - 1),
              (unsigned long long)__double_as_longlong(m));
  }
}

inline int blocks_for(long long work) { return (int)((work + kBlock - 1) / kBlock); }

}  // namespace

void launch_cfl_all(const GridParams &g, StepCtl *ctl, float *w0, float *w1, cudaStream_t st) {
  k_cfl<<<blocks_for(g.n), kBlock, 0, st>>>(g, ctl, w0, w1, 0);
}

void launch_cfl_margin(const GridParams &g, StepCtl *ctl, float *w0, float *w1, cudaStream_t st) {
  const long long work = margin::margin_cfl_cells(g);
  if (work > 0) k_cfl<<<blocks_for(work), kBlock, 0, st>>>(g, ctl, w0, w1, 1);
}

void launch_fill(const GridParams &g, StepCtl *ctl, float *w0, float *w1, cudaStream_t st) {
  if (g.my > 0) k_fill_y<<<blocks_for((long long)g.sx * g.my * g.sz), kBlock, 0, st>>>(g, ctl, w0, w1);
  if (g.mz > 0) k_fill_z<<<blocks_for((long long)g.sx * g.sy * g.mz), kBlock, 0, st>>>(g, ctl, w0, w1);
}

void launch_fill_predictor(const GridParams &g, StepCtl *ctl, float *wp, cudaStream_t st) {
  if (g.my > 0) k_fill_predictor_y<<<blocks_for((long long)g.sx * g.my * g.sz), kBlock, 0, st>>>(g, ctl, wp);
  if (g.mz > 0) k_fill_predictor_z<<<blocks_for((long long)g.sx * g.sy * g.mz), kBlock, 0, st>>>(g, ctl, wp);
}

void launch_halo_pack(const GridParams &g, StepCtl *ctl, const float *w0, const float *w1, float *send_inc,
                      float *send_dec, cudaStream_t st) {
  if (g.my > 0)
    k_halo_pack<<<blocks_for((long long)g.sx * g.my * g.sz), kBlock, 0, st>>>(g, ctl, w0, w1, send_inc, send_dec);
}

void launch_halo_unpack(const GridParams &g, StepCtl *ctl, float *w0, float *w1, const float *recv_inc,
                        const float *recv_dec, cudaStream_t st) {
  if (g.my > 0)
    k_halo_unpack<<<blocks_for((long long)g.sx * g.my * g.sz), kBlock, 0, st>>>(g, ctl, w0, w1, recv_inc,
                                                                              recv_dec);
  if (g.mz > 0) k_fill_z<<<blocks_for((long long)g.sx * g.sy * g.mz), kBlock, 0, st>>>(g, ctl, w0, w1);
}

void launch_cfl_min(const CflSlots &slots, cudaStream_t st) { k_cfl_min<<<1, 32, 0, st>>>(slots); }

void launch_flux(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                 int in_sel, int half, cudaStream_t st) {
  k_flux<<<blocks_for(g.n), kBlock, 0, st>>>(g, ctl, w0, w1, wp, flux, in_sel, half);
}

void launch_update(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                   float *dt_hist, int in_sel, int out_sel, int half, int final_stage, cudaStream_t st) {
  k_update<<<blocks_for(g.n), kBlock, 0, st>>>(g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel,
                                               half, final_stage);
}

void launch_stage(const GridParams &g, StepCtl *ctl, float *w0, float *w1, float *wp, float *flux,
                  float *dt_hist, int in_sel, int out_sel, int half, int final_stage, cudaStream_t st) {
  launch_flux(g, ctl, w0, w1, wp, flux, in_sel, half, st);
  launch_update(g, ctl, w0, w1, wp, flux, dt_hist, in_sel, out_sel, half, final_stage, st);
}

void launch_diag(const GridParams &g, StepCtl *ctl, float *w0, float *w1, double *acc, cudaStream_t st) {
  k_diag<<<blocks_for(g.n), kBlock, 0, st>>>(g, ctl, w0, w1, acc);
}

}  // namespace nmhd
