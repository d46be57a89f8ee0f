/* Body of the oracle (TEST INFRASTRUCTURE ONLY), included twice by
 * mhd_oracle.c: once with real = float (the reference's FP32 build) and once
 * with real = double (the reference with Real = double).
 *
 * Every expression keeps the reference's evaluation order and its implicit
 * float->double promotions (double literals such as 0.5*, 1.0/, 2.0*); the
 * library is compiled with -ffp-contract=off, so each operation rounds once,
 * as the reference's host build does.
 *
 * Required macros: real, FN(name), R_SQRT, R_FABS, R_FMAX, R_FMIN.
 */

/* ---- grid addressing ------------------------------------------------------
 * RCo<Bit> with CRYSTAL_PERIODIC_{X,Y,Z} (src/library/crystal.hrb:17-67):
 * address (z*Sy + y)*Sx + x with every coordinate wrapped periodically. */
typedef struct FN(grid) {
  int sx, sy, sz;
  size_t n;
} FN(grid);

static inline size_t FN(at)(const FN(grid) *g, int x, int y, int z) {
  x = (x % g->sx + g->sx) % g->sx;
  y = (y % g->sy + g->sy) % g->sy;
  z = (z % g->sz + g->sz) % g->sz;
  return ((size_t)z * g->sy + y) * g->sx + x;
}
/* address of (c + off) where off is along axis a by da */
static inline size_t FN(at3)(const FN(grid) *g, const int c[3], int a, int da, int b, int db) {
  int p[3] = {c[0], c[1], c[2]};
  p[a] += da;
  p[b] += db;
  return FN(at)(g, p[0], p[1], p[2]);
}

/* ---- derived constants (simulation_config_default.h:56-103) -------------- */
typedef struct FN(consts) {
  real d[3];        /* kDX, kDY, kDZ */
  real corner_y;    /* -gExtentY/2: origin of the Kepler local coordinate */
  real gamma, cfl, q, omega;
  double rel_vel;   /* relative_velocity(): -q*Omega*kLocalExtentY */
  real extent_x;    /* kExtentX */
} FN(consts);

static void FN(derive)(const oracle_config *c, FN(consts) *k) {
  int s[3] = {c->size_x, c->size_y, c->size_z};
  /* kLocalSize (interior of this rank) and kGlobalSize (P ranks along Y) */
  const int py = c->parallel_size_y > 1 ? c->parallel_size_y : 1;
  int lsz[3] = {c->size_x, c->size_y - 2 * c->margin_y, c->size_z - 2 * c->margin_z};
  int gsz[3] = {lsz[0], py * lsz[1], lsz[2]};
  float ext[3] = {c->extent_x, c->extent_y, c->extent_z};
  real comp_ext[3], local_ext[3];
  for (int i = 0; i < 3; ++i) {
    real L = (real)ext[i];
    comp_ext[i] = (real)((real)(L / (real)gsz[i]) * (real)s[i]);
    local_ext[i] = (real)((real)(L / (real)gsz[i]) * (real)lsz[i]);
    k->d[i] = comp_ext[i] / (real)s[i];
  }
  k->extent_x = comp_ext[0];
  k->corner_y = -comp_ext[1] / 2;
  k->gamma = (real)c->gamma;
  k->cfl = (real)c->cfl;
  k->q = (real)c->q;
  k->omega = (real)c->omega;
  /* relative_velocity() hook: the Kepler app's (kepler_disk_demo/mhd_solver.curb:50-52),
     zero without a shearing box */
  k->rel_vel = c->problem == 1 ? (double)((real)(-k->q * k->omega) * local_ext[1]) : 0.0;
}

/* ---- minbee reconstruction (src/library/mhd_solver.inlrb:140-155) -------- */
static inline real FN(absolute_smaller)(real a, real b) {
  return a * b <= 0 ? 0 : R_FABS(a) < R_FABS(b) ? a : b;
}
static inline void FN(interpolate4)(real x0, real x1, real x2, real x3, real *l, real *r) {
  real d01 = x1 - x0, d12 = x2 - x1, d23 = x3 - x2;
  real d1 = FN(absolute_smaller)(d01, d12);
  real d2 = FN(absolute_smaller)(d12, d23);
  *l = x1 + d1 / 2;
  *r = x2 - d2 / 2;
}

/* ---- HLLD flux (src/library/hlld.inl:7-284, the `#if 1` wave speeds) ----- */
void FN(oracle_hlld)(real gamma, real Bx, const real lr[14], real out[7]) {
  const real dens_L = lr[0], dens_R = lr[1], velx_L = lr[2], velx_R = lr[3];
  const real vely_L = lr[4], vely_R = lr[5], velz_L = lr[6], velz_R = lr[7];
  const real pres_L = lr[8], pres_R = lr[9], By_L = lr[10], By_R = lr[11];
  const real Bz_L = lr[12], Bz_R = lr[13];
  const real TINY = (real)1.0e-10;
  real signBx = 0;
  if (R_FABS(Bx) > 0) signBx = Bx / R_FABS(Bx);
  real momx_L = dens_L * velx_L, momy_L = dens_L * vely_L, momz_L = dens_L * velz_L;
  real momx_R = dens_R * velx_R, momy_R = dens_R * vely_R, momz_R = dens_R * velz_R;
  real B2_L = Bx * Bx + By_L * By_L + Bz_L * Bz_L;
  real v2_L = velx_L * velx_L + vely_L * vely_L + velz_L * velz_L;
  real etot_L = (real)((double)(pres_L / (gamma - 1)) + 0.5 * (double)dens_L * (double)v2_L +
                       0.5 * (double)B2_L);
  real B2_R = Bx * Bx + By_R * By_R + Bz_R * Bz_R;
  real v2_R = velx_R * velx_R + vely_R * vely_R + velz_R * velz_R;
  real etot_R = (real)((double)(pres_R / (gamma - 1)) + 0.5 * (double)dens_R * (double)v2_R +
                       0.5 * (double)B2_R);
  real gpl = gamma * pres_L, gpr = gamma * pres_R;
  real gpbl = gpl + B2_L, gpbr = gpr + B2_R;
  const float fsig = (float)sqrt(2.0);
  real cfl = R_SQRT((real)((double)(gpbl + R_SQRT(gpbl * gpbl - 4 * gpl * (Bx * Bx))) /
                           (2.0 * (double)dens_L)));
  real cfr = R_SQRT((real)((double)(gpbr + R_SQRT(gpbr * gpbr - 4 * gpr * (Bx * Bx))) /
                           (2.0 * (double)dens_R)));
  real cfmax = fsig * R_FMAX(cfl, cfr);
  real S_L = R_FMIN(velx_L, velx_R) - cfmax;
  real S_R = R_FMAX(velx_L, velx_R) + cfmax;

  real pT_L = (real)((double)pres_L + 0.5 * (double)B2_L);
  real pT_R = (real)((double)pres_R + 0.5 * (double)B2_R);
  real S_M = (S_R - velx_R) * momx_R - (S_L - velx_L) * momx_L - pT_R + pT_L;
  real den = (S_R - velx_R) * dens_R - (S_L - velx_L) * dens_L;
  S_M = (real)((double)S_M * (1.0 / (double)den));
  real pT_s = (S_R - velx_R) * dens_R * pT_L - (S_L - velx_L) * dens_L * pT_R;
  pT_s = pT_s + dens_L * dens_R * (S_R - velx_R) * (S_L - velx_L) * (velx_R - velx_L);
  pT_s = (real)((double)pT_s * (1.0 / (double)den));

  real B2x = Bx * Bx;
  real dens_L_s = dens_L * (S_L - velx_L) / (S_L - S_M);
  real dnL = dens_L * (S_L - velx_L) * (S_L - S_M) - B2x + TINY;
  real vely_L_s = vely_L - Bx * By_L * (S_M - velx_L) / dnL;
  real velz_L_s = velz_L - Bx * Bz_L * (S_M - velx_L) / dnL;
  real tL = S_L - velx_L;
  real By_L_s = By_L * (dens_L * (tL * tL) - B2x) / dnL;
  real Bz_L_s = Bz_L * (dens_L * (tL * tL) - B2x) / dnL;

  real dens_R_s = dens_R * (S_R - velx_R) / (S_R - S_M);
  real dnR = dens_R * (S_R - velx_R) * (S_R - S_M) - B2x + TINY;
  real vely_R_s = vely_R - Bx * By_R * (S_M - velx_R) / dnR;
  real velz_R_s = velz_R - Bx * Bz_R * (S_M - velx_R) / dnR;
  real tR = S_R - velx_R;
  real By_R_s = By_R * (dens_R * (tR * tR) - B2x) / dnR;
  real Bz_R_s = Bz_R * (dens_R * (tR * tR) - B2x) / dnR;

  real vB_L = velx_L * Bx + vely_L * By_L + velz_L * Bz_L;
  real vB_L_s = S_M * Bx + vely_L_s * By_L_s + velz_L_s * Bz_L_s;
  real etot_L_s =
      ((S_L - velx_L) * etot_L - pT_L * velx_L + pT_s * S_M + Bx * (vB_L - vB_L_s)) / (S_L - S_M);
  real vB_R = velx_R * Bx + vely_R * By_R + velz_R * Bz_R;
  real vB_R_s = S_M * Bx + vely_R_s * By_R_s + velz_R_s * Bz_R_s;
  real etot_R_s =
      ((S_R - velx_R) * etot_R - pT_R * velx_R + pT_s * S_M + Bx * (vB_R - vB_R_s)) / (S_R - S_M);

  real sdL = R_SQRT(dens_L_s), sdR = R_SQRT(dens_R_s);
  real S_L_s = S_M - R_FABS(Bx) / sdL;
  real S_R_s = S_M + R_FABS(Bx) / sdR;
  real f = (real)(1.0 / (double)(sdL + sdR));
  real vely_ss = f * (sdL * vely_L_s + sdR * vely_R_s + (By_R_s - By_L_s) * signBx);
  real velz_ss = f * (sdL * velz_L_s + sdR * velz_R_s + (Bz_R_s - Bz_L_s) * signBx);
  real sdLR = R_SQRT(dens_L_s * dens_R_s);
  real By_ss = f * (sdL * By_R_s + sdR * By_L_s + sdLR * (vely_R_s - vely_L_s) * signBx);
  real Bz_ss = f * (sdL * Bz_R_s + sdR * Bz_L_s + sdLR * (velz_R_s - velz_L_s) * signBx);
  real vB_ss = S_M * Bx + vely_ss * By_ss + velz_ss * Bz_ss;
  real etot_L_ss = etot_L_s - sdL * (vB_L_s - vB_ss) * signBx;
  real etot_R_ss = etot_R_s + sdR * (vB_R_s - vB_ss) * signBx;

  real FL[7] = {dens_L * velx_L, momx_L * velx_L + pT_L - B2x, momy_L * velx_L - Bx * By_L,
                momz_L * velx_L - Bx * Bz_L, etot_L * velx_L + pT_L * velx_L - Bx * vB_L,
                By_L * velx_L - Bx * vely_L, Bz_L * velx_L - Bx * velz_L};
  real FR[7] = {dens_R * velx_R, momx_R * velx_R + pT_R - B2x, momy_R * velx_R - Bx * By_R,
                momz_R * velx_R - Bx * Bz_R, etot_R * velx_R + pT_R * velx_R - Bx * vB_R,
                By_R * velx_R - Bx * vely_R, Bz_R * velx_R - Bx * velz_R};
  real UL[7] = {dens_L, momx_L, momy_L, momz_L, etot_L, By_L, Bz_L};
  real UR[7] = {dens_R, momx_R, momy_R, momz_R, etot_R, By_R, Bz_R};
  real ULs[7] = {dens_L_s, dens_L_s * S_M, dens_L_s * vely_L_s, dens_L_s * velz_L_s,
                 etot_L_s, By_L_s, Bz_L_s};
  real URs[7] = {dens_R_s, dens_R_s * S_M, dens_R_s * vely_R_s, dens_R_s * velz_R_s,
                 etot_R_s, By_R_s, Bz_R_s};
  real ULss[7] = {dens_L_s, dens_L_s * S_M, dens_L_s * vely_ss, dens_L_s * velz_ss,
                  etot_L_ss, By_ss, Bz_ss};
  real URss[7] = {dens_R_s, dens_R_s * S_M, dens_R_s * vely_ss, dens_R_s * velz_ss,
                  etot_R_ss, By_ss, Bz_ss};
  for (int i = 0; i < 7; ++i) {
    if (S_L > 0) {
      out[i] = FL[i];
    } else if (S_L <= 0 && 0 <= S_L_s) {
      out[i] = FL[i] + S_L * ULs[i] - S_L * UL[i];
    } else if (S_L_s <= 0 && 0 <= S_M) {
      out[i] = FL[i] + S_L_s * ULss[i] - (S_L_s - S_L) * ULs[i] - S_L * UL[i];
    } else if (S_M <= 0 && 0 <= S_R_s) {
      out[i] = FR[i] + S_R_s * URss[i] - (S_R_s - S_R) * URs[i] - S_R * UR[i];
    } else if (S_R_s <= 0 && 0 <= S_R) {
      out[i] = FR[i] + S_R * URs[i] - S_R * UR[i];
    } else {
      out[i] = FR[i];
    }
  }
}

/* ---- solver state --------------------------------------------------------- */
typedef struct FN(solver) {
  oracle_config cfg;
  FN(grid) g;
  FN(consts) k;
  real *w;    /* 8 fields: rho vx vy vz p Bx By Bz */
  real *wp;   /* predictor, same layout */
  real *mom;  /* 3 fields: conserved momentum scratch */
  real *ene;  /* conserved energy scratch */
  real *pace; /* 8 fields: d/dt of rho, m, E, B */
  real *flux; /* 7 fields of the current sweep */
} FN(solver);

#define F_RHO 0
#define F_VX 1
#define F_P 4
#define F_BX 5

static inline real *FN(fld)(real *base, size_t n, int i) { return base + (size_t)i * n; }

/* Kepler acceleration (src/application/kepler_disk_demo/mhd_solver.curb:57-86)
 * for velocity (vX, vY) at radial index y; RCo::position adds half a cell for
 * every staggering (crystal.hrb:55-62: `Bit & mask == 0` is always false). */
static inline real FN(ly)(const FN(consts) *k, int yw) {
  return k->corner_y + k->d[1] * ((real)yw + (real)0.5f);
}
static inline void FN(kepler)(const FN(consts) *k, real vX, real vY, int yw, real a[3]) {
  a[0] = -(real)2.0 * k->omega * vY;
  a[1] = (real)2.0 * k->omega * vX + (real)2.0 * k->q * (k->omega * k->omega) * FN(ly)(k, yw);
  a[2] = 0;
}

/* calc_flux_kernel<EX> (src/library/mhd_solver.inlrb:562-636): flux through
 * the lower ex-face of every cell. */
static void FN(calc_flux)(FN(solver) *s, int ex, real dt, real *w) {
  const FN(grid) *g = &s->g;
  const size_t n = g->n;
  const int ey = (ex + 1) % 3, ez = (ex + 2) % 3;
  const int order2 = s->cfg.space_order != 1;
  const int shear = s->cfg.problem == 1;
  real *rho = FN(fld)(w, n, F_RHO), *p = FN(fld)(w, n, F_P);
  real *vex = FN(fld)(w, n, F_VX + ex), *vey = FN(fld)(w, n, F_VX + ey), *vez = FN(fld)(w, n, F_VX + ez);
  real *bex = FN(fld)(w, n, F_BX + ex), *bey = FN(fld)(w, n, F_BX + ey), *bez = FN(fld)(w, n, F_BX + ez);
  real *fl = s->flux;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < g->sz; ++z)
    for (int y = 0; y < g->sy; ++y)
      for (int x = 0; x < g->sx; ++x) {
        const int c[3] = {x, y, z};
        size_t id[4];
        for (int t = 0; t < 4; ++t) id[t] = FN(at3)(g, c, ex, t - 2, ey, 0);
        real lr[14];
        real *vars[5] = {rho, vex, vey, vez, p};
        for (int v = 0; v < 5; ++v) {
          if (order2)
            FN(interpolate4)(vars[v][id[0]], vars[v][id[1]], vars[v][id[2]], vars[v][id[3]],
                             &lr[2 * v], &lr[2 * v + 1]);
          else {
            lr[2 * v] = vars[v][id[1]];
            lr[2 * v + 1] = vars[v][id[2]];
          }
        }
        real avg_y[4], avg_z[4];
        for (int t = 0; t < 4; ++t) {
          int cc[3] = {c[0], c[1], c[2]};
          cc[ex] += t - 2;
          avg_y[t] = (real)0.5f * (bey[FN(at)(g, cc[0], cc[1], cc[2])] + bey[FN(at3)(g, cc, ey, 1, ex, 0)]);
          avg_z[t] = (real)0.5f * (bez[FN(at)(g, cc[0], cc[1], cc[2])] + bez[FN(at3)(g, cc, ez, 1, ex, 0)]);
        }
        if (order2) {
          FN(interpolate4)(avg_y[0], avg_y[1], avg_y[2], avg_y[3], &lr[10], &lr[11]);
          FN(interpolate4)(avg_z[0], avg_z[1], avg_z[2], avg_z[3], &lr[12], &lr[13]);
        } else {
          lr[10] = avg_y[1]; lr[11] = avg_y[2];
          lr[12] = avg_z[1]; lr[13] = avg_z[2];
        }
        if (shear) {
          /* face-centred acceleration: velocities averaged across the face */
          real *vx = FN(fld)(w, n, F_VX), *vy = FN(fld)(w, n, F_VX + 1);
          real vX = (real)0.5f * (vx[id[1]] + vx[id[2]]);
          real vY = (real)0.5f * (vy[id[1]] + vy[id[2]]);
          real a[3];
          FN(kepler)(&s->k, vX, vY, y, a);
          real mbv = (real)0.5 * dt * a[ex];
          lr[2] += mbv;
          lr[3] += mbv;
        }
        real out[7];
        size_t o = FN(at)(g, x, y, z);
        FN(oracle_hlld)(s->k.gamma, bex[o], lr, out);
        for (int v = 0; v < 7; ++v) fl[(size_t)v * n + o] = out[v];
      }
}

/* corner_magnet_flux (src/library/mhd_solver.inlrb:641-653): the ea-flux of
 * B_eb at the edge with lower-face indices c in ea and eb. */
static inline real FN(corner)(const FN(grid) *g, const int c[3], int ea, int eb, const real *wind_b,
                              const real *flux_b) {
  real w = wind_b[FN(at3)(g, c, ea, 0, eb, 0)] + wind_b[FN(at3)(g, c, ea, 0, eb, -1)] +
           wind_b[FN(at3)(g, c, ea, -1, eb, 0)] + wind_b[FN(at3)(g, c, ea, -1, eb, -1)];
  real f0 = flux_b[FN(at3)(g, c, eb, -1, ea, 0)];
  real f1 = flux_b[FN(at3)(g, c, eb, 0, ea, 0)];
  return w > 0 ? f0 : w < 0 ? f1 : (real)0.5f * (f0 + f1);
}
/* magnet_flux_difference (mhd_solver.inlrb:659-666) across axis h */
static inline real FN(mfd)(const FN(grid) *g, const int c[3], int ea, int eb, int h,
                           const real *wind_b, const real *flux_b) {
  int up[3] = {c[0], c[1], c[2]};
  up[h] += 1;
  return FN(corner)(g, up, ea, eb, wind_b, flux_b) - FN(corner)(g, c, ea, eb, wind_b, flux_b);
}

/* add_flux_kernel<EX> (mhd_solver.inlrb:668-714) */
static void FN(add_flux)(FN(solver) *s, int ex, real *wind) {
  const FN(grid) *g = &s->g;
  const size_t n = g->n;
  const int ey = (ex + 1) % 3, ez = (ex + 2) % 3;
  const real *d = s->k.d;
  const real magic = (real)0.5f, black_magic = (real)1.0f;
  real *fl = s->flux, *pace = s->pace;
  /* flux component -> pace field: rho, m_ex, m_ey, m_ez, E */
  const int target[5] = {0, 1 + ex, 1 + ey, 1 + ez, 4};
  const real *fb_ey = fl + 5 * n, *fb_ez = fl + 6 * n;
  const real *w_ey = FN(fld)(wind, n, F_VX + ey), *w_ez = FN(fld)(wind, n, F_VX + ez);
#pragma omp parallel for schedule(static)
  for (int z = 0; z < g->sz; ++z)
    for (int y = 0; y < g->sy; ++y)
      for (int x = 0; x < g->sx; ++x) {
        const int c[3] = {x, y, z};
        size_t o = FN(at)(g, x, y, z);
        size_t up = FN(at3)(g, c, ex, 1, ey, 0);
        for (int v = 0; v < 5; ++v) {
          const real *f = fl + (size_t)v * n;
          real *pc = pace + (size_t)target[v] * n;
          pc[o] += (f[o] - f[up]) / d[ex];
        }
        real *pb_ex = pace + (size_t)(5 + ex) * n, *pb_ey = pace + (size_t)(5 + ey) * n,
             *pb_ez = pace + (size_t)(5 + ez) * n;
        pb_ey[o] -= magic * FN(mfd)(g, c, ex, ey, ex, w_ey, fb_ey) / d[ex];
        pb_ez[o] -= magic * FN(mfd)(g, c, ex, ez, ex, w_ez, fb_ez) / d[ex];
        pb_ex[o] += magic * black_magic *
                    (FN(mfd)(g, c, ex, ey, ey, w_ey, fb_ey) / d[ey] +
                     FN(mfd)(g, c, ex, ez, ez, w_ez, fb_ez) / d[ez]);
      }
}

/* to_conserved_kernel (mhd_solver.inlrb:762-777) */
static void FN(to_conserved)(FN(solver) *s, real *w) {
  const FN(grid) *g = &s->g;
  const size_t n = g->n;
  const real gm1 = s->k.gamma - 1;
  real *rho = w, *p = w + 4 * n;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < g->sz; ++z)
    for (int y = 0; y < g->sy; ++y)
      for (int x = 0; x < g->sx; ++x) {
        const int c[3] = {x, y, z};
        size_t o = FN(at)(g, x, y, z);
        real v[3], b2[6];
        for (int a = 0; a < 3; ++a) {
          v[a] = w[(size_t)(1 + a) * n + o];
          s->mom[(size_t)a * n + o] = rho[o] * v[a];
          real *b = w + (size_t)(5 + a) * n;
          real lo = b[o], hi = b[FN(at3)(g, c, a, 1, a, 0)];
          b2[2 * a] = lo * lo;
          b2[2 * a + 1] = hi * hi;
        }
        s->ene[o] = p[o] / gm1 + (real)0.5f * rho[o] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) +
                    (real)0.25f * (b2[0] + b2[1] + b2[2] + b2[3] + b2[4] + b2[5]);
      }
}

/* add_pace_kernel / update_kernel (mhd_solver.inlrb:797-835):
 * rho_out = rho_bef + dt*pace, m,E += dt*pace, B_out = B_bef + dt*pace */
static void FN(add_pace)(FN(solver) *s, real dt, const real *bef, real *out) {
  const size_t n = s->g.n;
#pragma omp parallel for schedule(static)
  for (size_t o = 0; o < n; ++o) {
    out[o] = bef[o] + dt * s->pace[o];
    for (int a = 0; a < 3; ++a) s->mom[a * n + o] += dt * s->pace[(1 + a) * n + o];
    s->ene[o] += dt * s->pace[4 * n + o];
    for (int a = 0; a < 3; ++a) out[(5 + a) * n + o] = bef[(5 + a) * n + o] + dt * s->pace[(5 + a) * n + o];
  }
}

/* to_primitive_kernel (mhd_solver.inlrb:779-795) */
static void FN(to_primitive)(FN(solver) *s, real *w) {
  const FN(grid) *g = &s->g;
  const size_t n = g->n;
  const real gm1 = s->k.gamma - 1;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < g->sz; ++z)
    for (int y = 0; y < g->sy; ++y)
      for (int x = 0; x < g->sx; ++x) {
        const int c[3] = {x, y, z};
        size_t o = FN(at)(g, x, y, z);
        real rho = w[o], m[3], b2[6];
        for (int a = 0; a < 3; ++a) {
          m[a] = s->mom[(size_t)a * n + o];
          w[(size_t)(1 + a) * n + o] = m[a] / rho;
          real *b = w + (size_t)(5 + a) * n;
          real lo = b[o], hi = b[FN(at3)(g, c, a, 1, a, 0)];
          b2[2 * a] = lo * lo;
          b2[2 * a + 1] = hi * hi;
        }
        real internal = s->ene[o] - (real)0.5f * (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) / rho -
                        (real)0.25f * (b2[0] + b2[1] + b2[2] + b2[3] + b2[4] + b2[5]);
        w[4 * n + o] = internal * gm1;
      }
}

/* external_acceleration_kernel (mhd_solver.inlrb:837-848) with the Kepler
 * hook: a from the cell's own velocity, then v += dt*a. */
static void FN(kick)(FN(solver) *s, real dt, real *w) {
  const FN(grid) *g = &s->g;
  const size_t n = g->n;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < g->sz; ++z)
    for (int y = 0; y < g->sy; ++y)
      for (int x = 0; x < g->sx; ++x) {
        size_t o = FN(at)(g, x, y, z);
        real a[3];
        FN(kepler)(&s->k, w[n + o], w[2 * n + o], y, a);
        for (int d = 0; d < 3; ++d) w[(size_t)(1 + d) * n + o] += dt * a[d];
      }
}

/* cfl_condition_kernel + min_element (mhd_solver.inlrb:496-521, 870-879) */
static real FN(cfl_min)(const oracle_config *cfg, const FN(grid) *g, const FN(consts) *k,
                        const real *w, real goal) {
  const size_t n = g->n;
  real best = goal;
#pragma omp parallel for schedule(static) reduction(min : best)
  for (int z = 0; z < g->sz; ++z)
    for (int y = 0; y < g->sy; ++y)
      for (int x = 0; x < g->sx; ++x) {
        const int c[3] = {x, y, z};
        size_t o = FN(at)(g, x, y, z);
        real b2 = 0;
        for (int a = 0; a < 3; ++a) {
          const real *b = w + (size_t)(5 + a) * n;
          real lo = b[o], hi = b[FN(at3)(g, c, a, 1, a, 0)];
          real m = R_FMAX(lo * lo, hi * hi);
          b2 = a == 0 ? m : b2 + m;
        }
        real t = goal;
        for (int a = 0; a < 3; ++a) {
          real speed = R_FABS(w[(size_t)(1 + a) * n + o] + R_SQRT((k->gamma * w[4 * n + o] + b2) / w[o]));
          t = R_FMIN(t, k->cfl * k->d[a] / speed);
        }
        if (t < best) best = t;
      }
  (void)cfg;
  return best;
}

/* relative_displacement (mhd_solver.inlrb:244-259) for one rank */
static void FN(displacement)(const FN(consts) *k, double t, int *d_int, real *minor) {
  double displacement0 = 0.0 + t * k->rel_vel;
  int folding_number = (int)floor(displacement0 / (double)k->extent_x);
  double displacement1 = displacement0 - (double)((real)folding_number * k->extent_x);
  *d_int = (int)floor(displacement1 / (double)k->d[0]);
  *minor = (real)(displacement1 / (double)k->d[0] - *d_int);
}

/* communicate_gather_kernel_y (mhd_solver.inlrb:184-222): the two outgoing
 * messages of the Y-margin exchange at time t, item (z*M + y)*Sx + x of
 * field v at v*unit + item: buf_inc (to the rank above) from the top interior
 * rows shifted by +d_int, v_X - relative_velocity; buf_dec (to the rank below)
 * from the bottom interior rows shifted by -d_int-1, v_X + relative_velocity.
 * The interpolation weights both multiply the same sample, as the
 * reference's do. */
static void FN(halo_pack)(const oracle_config *cfg, const FN(grid) *g, const FN(consts) *k, const real *w,
                          double t, real *buf_inc, real *buf_dec) {
  const int M = cfg->margin_y;
  const int sx = g->sx, sy = g->sy, sz = g->sz;
  const size_t n = g->n;
  int d_int;
  real f;
  FN(displacement)(k, t, &d_int, &f);
  const real rv = (real)k->rel_vel;
  const size_t unit = (size_t)sx * M * sz;
  for (int v = 0; v < 8; ++v) {
    const real *var = w + (size_t)v * n;
#pragma omp parallel for schedule(static)
    for (int zz = 0; zz < sz; ++zz)
      for (int yy = 0; yy < M; ++yy)
        for (int xx = 0; xx < sx; ++xx) {
          size_t a = ((size_t)zz * M + yy) * sx + xx;
          int inc_x0 = (xx + d_int) % sx;
          int dec_x0 = (xx - d_int - 1 + sx) % sx;
          real vi = var[((size_t)zz * sy + (sy - 2 * M + yy)) * sx + inc_x0];
          real vd = var[((size_t)zz * sy + (M + yy)) * sx + dec_x0];
          real bi = ((real)1 - f) * vi + f * vi;
          real bd = f * vd + ((real)1 - f) * vd;
          if (v == F_VX) {
            bi = bi - rv;
            bd = bd + rv;
          }
          buf_inc[(size_t)v * unit + a] = bi;
          buf_dec[(size_t)v * unit + a] = bd;
        }
  }
}

/* communicate_scatter_kernel_y (mhd_solver.inlrb:224-242): the message from
 * the rank below (recv_inc) into the bottom margin, the one from the rank
 * above (recv_dec) into the top margin except By of its first row; then the
 * plain Z-margin copies (:384-402, 463-480). */
static void FN(halo_unpack)(const oracle_config *cfg, const FN(grid) *g, real *w, const real *recv_inc,
                            const real *recv_dec) {
  const int M = cfg->margin_y, Mz = cfg->margin_z;
  const int sx = g->sx, sy = g->sy, sz = g->sz;
  const size_t n = g->n;
  if (M > 0) {
    const size_t unit = (size_t)sx * M * sz;
    for (int v = 0; v < 8; ++v) {
      real *var = w + (size_t)v * n;
#pragma omp parallel for schedule(static)
      for (int zz = 0; zz < sz; ++zz)
        for (int yy = 0; yy < M; ++yy)
          for (int xx = 0; xx < sx; ++xx) {
            size_t a = ((size_t)zz * M + yy) * sx + xx;
            var[((size_t)zz * sy + yy) * sx + xx] = recv_inc[(size_t)v * unit + a];
            if (!(v == F_BX + 1 && yy == 0))
              var[((size_t)zz * sy + (sy - M + yy)) * sx + xx] = recv_dec[(size_t)v * unit + a];
          }
    }
  }
  if (Mz > 0) {
    const size_t unit = (size_t)sx * sy * Mz;
    for (int v = 0; v < 8; ++v) {
      real *var = w + (size_t)v * n;
      real *inc = (real *)malloc(sizeof(real) * unit), *dec = (real *)malloc(sizeof(real) * unit);
      memcpy(inc, var + (n - 2 * unit), sizeof(real) * unit);
      memcpy(dec, var + unit, sizeof(real) * unit);
      memcpy(var, inc, sizeof(real) * unit);
      memcpy(var + (n - unit), dec, sizeof(real) * unit);
      free(inc);
      free(dec);
    }
  }
}

/* communicate() with one rank (mhd_solver.inlrb:283-493): each message
 * delivered to the rank itself (the single box's shear-periodic boundary). */
static void FN(shear_fill_impl)(const oracle_config *cfg, const FN(grid) *g, const FN(consts) *k,
                                real *w, double t) {
  const size_t unit = (size_t)g->sx * cfg->margin_y * g->sz;
  real *buf_inc = NULL, *buf_dec = NULL;
  if (cfg->margin_y > 0) {
    buf_inc = (real *)malloc(sizeof(real) * unit * 8);
    buf_dec = (real *)malloc(sizeof(real) * unit * 8);
    FN(halo_pack)(cfg, g, k, w, t, buf_inc, buf_dec);
  }
  FN(halo_unpack)(cfg, g, w, buf_inc, buf_dec);
  free(buf_inc);
  free(buf_dec);
}

/* one integrator stage (mhd_solver.inlrb:908-962):
 * fluxes from w_in (wind = its velocity), U from w_bef, result in w_out */
static void FN(stage)(FN(solver) *s, real dt, real *w_in, real *w_bef, real *w_out) {
  const size_t n = s->g.n;
  memset(s->pace, 0, sizeof(real) * 8 * n);
  for (int ex = 0; ex < 3; ++ex) {
    FN(calc_flux)(s, ex, dt, w_in);
    FN(add_flux)(s, ex, w_in);
  }
  FN(to_conserved)(s, w_bef);
  FN(add_pace)(s, dt, w_bef, w_out);
  FN(to_primitive)(s, w_out);
  if (s->cfg.problem == 1) FN(kick)(s, dt, w_out);
}

/* The RK stages of one step with time step dt from time t (mhd_solver.inlrb:966-975) */
static void FN(run_stages)(FN(solver) *s, real dt, double t) {
  if (s->cfg.time_order == 1) {
    FN(stage)(s, dt, s->w, s->w, s->w);
  } else {
    FN(stage)(s, dt / 2, s->w, s->w, s->wp);
    /* nmhd_config flag HALO_PER_STAGE (no reference counterpart): the
       predictor's margins refilled at its time t + dt/2 */
    if (s->cfg.flags & 1) FN(shear_fill_impl)(&s->cfg, &s->g, &s->k, s->wp, t + (double)(dt / 2));
    FN(stage)(s, dt, s->wp, s->w, s->w);
  }
}

/* MHDSolver::proceed (mhd_solver.inlrb:850-993) for at most max_steps steps */
int FN(oracle_proceed)(const oracle_config *cfg, real *state, double *time, int64_t *generation,
                       double goal_time, int max_steps, double *times_out, real *dt_out,
                       int *goal_reached) {
  FN(solver) s;
  s.cfg = *cfg;
  s.g.sx = cfg->size_x;
  s.g.sy = cfg->size_y;
  s.g.sz = cfg->size_z;
  s.g.n = (size_t)cfg->size_x * cfg->size_y * cfg->size_z;
  FN(derive)(cfg, &s.k);
  const size_t n = s.g.n;
  s.w = state;
  s.wp = (real *)calloc(8 * n, sizeof(real));
  s.mom = (real *)calloc(3 * n, sizeof(real));
  s.ene = (real *)calloc(n, sizeof(real));
  s.pace = (real *)calloc(8 * n, sizeof(real));
  s.flux = (real *)calloc(7 * n, sizeof(real));
  const real goal = (real)goal_time;
  int steps = 0;
  int done = 0;
  while (!done && steps < max_steps) {
    if (times_out) times_out[steps] = *time;
    FN(shear_fill_impl)(cfg, &s.g, &s.k, s.w, *time);
    real dt = FN(cfl_min)(cfg, &s.g, &s.k, s.w, goal);
    if (dt < 0) break;
    double next_time = *time + (double)dt;
    if (next_time > (double)goal) {
      dt = (real)((double)goal - *time);
      done = 1;
    }
    if (dt_out) dt_out[steps] = dt;
    FN(run_stages)(&s, dt, *time);
    *time += (double)dt;
    *generation += 1;
    ++steps;
  }
  if (times_out) times_out[steps] = *time;
  free(s.wp);
  free(s.mom);
  free(s.ene);
  free(s.pace);
  free(s.flux);
  if (goal_reached) *goal_reached = done;
  return steps;
}

static void FN(setup)(const oracle_config *cfg, FN(grid) *g, FN(consts) *k) {
  g->sx = cfg->size_x;
  g->sy = cfg->size_y;
  g->sz = cfg->size_z;
  g->n = (size_t)cfg->size_x * cfg->size_y * cfg->size_z;
  FN(derive)(cfg, k);
}

real FN(oracle_cfl)(const oracle_config *cfg, const real *state, real goal) {
  FN(grid) g;
  FN(consts) k;
  FN(setup)(cfg, &g, &k);
  return FN(cfl_min)(cfg, &g, &k, state, goal);
}

void FN(oracle_shear_fill)(const oracle_config *cfg, real *state, double time) {
  FN(grid) g;
  FN(consts) k;
  FN(setup)(cfg, &g, &k);
  FN(shear_fill_impl)(cfg, &g, &k, state, time);
}

void FN(oracle_halo_pack)(const oracle_config *cfg, const real *state, double time, real *send_inc,
                          real *send_dec) {
  FN(grid) g;
  FN(consts) k;
  FN(setup)(cfg, &g, &k);
  if (cfg->margin_y > 0) FN(halo_pack)(cfg, &g, &k, state, time, send_inc, send_dec);
}

void FN(oracle_halo_unpack)(const oracle_config *cfg, real *state, const real *recv_inc,
                            const real *recv_dec) {
  FN(grid) g;
  FN(consts) k;
  FN(setup)(cfg, &g, &k);
  FN(halo_unpack)(cfg, &g, state, recv_inc, recv_dec);
}

void FN(oracle_stages)(const oracle_config *cfg, real *state, real dt) {
  FN(solver) s;
  s.cfg = *cfg;
  s.cfg.flags &= ~1;  /* a slab has no per-stage margin refill (nmhd_create refuses it) */
  FN(setup)(cfg, &s.g, &s.k);
  const size_t n = s.g.n;
  s.w = state;
  s.wp = (real *)calloc(8 * n, sizeof(real));
  s.mom = (real *)calloc(3 * n, sizeof(real));
  s.ene = (real *)calloc(n, sizeof(real));
  s.pace = (real *)calloc(8 * n, sizeof(real));
  s.flux = (real *)calloc(7 * n, sizeof(real));
  FN(run_stages)(&s, dt, 0.0);
  free(s.wp);
  free(s.mom);
  free(s.ene);
  free(s.pace);
  free(s.flux);
}
