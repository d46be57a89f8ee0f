// Device arithmetic of the ideal-MHD time step (sm_100a).
//
// Every function keeps the reference's evaluation order and its implicit
// float->double promotions, and the translation units that include this file
// are compiled with -fmad=false (no multiply-add contraction), so each float
// operation rounds exactly once, as in the reference.  IEEE division and square
// root (-prec-div=true, -prec-sqrt=true, no flush-to-zero) are the defaults.
//
// With NMHD_FAST_ARITH (the fast-arithmetic flux kernel, cell_fast.cu, compiled
// with contraction and approximate division and square root) the FP64
// sub-expressions are evaluated in float: results within the documented
// tolerance of the reference instead of bitwise.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nmhd {

// Minbee limiter: src/library/mhd_solver.inlrb:140-145.
__host__ __device__ __forceinline__ float absolute_smaller(float a, float b) {
  return a * b <= 0.0f ? 0.0f : (fabsf(a) < fabsf(b) ? a : b);
}

// 4-cell MUSCL reconstruction at the face between x1 and x2:
// src/library/mhd_solver.inlrb:147-155.
__host__ __device__ __forceinline__ void reconstruct4(float x0, float x1, float x2, float x3, float &left,
                                             float &right) {
  const float d01 = x1 - x0;
  const float d12 = x2 - x1;
  const float d23 = x3 - x2;
  const float d1 = absolute_smaller(d01, d12);
  const float d2 = absolute_smaller(d12, d23);
  left = x1 + d1 / 2.0f;
  right = x2 - d2 / 2.0f;
}

// HLLD flux, src/library/hlld.inl:7-284 (the `#if 1` fast-magnetosonic
// bounds).  Inputs: normal field bx and the left/right states
// (rho, v_n, v_t1, v_t2, p, B_t1, B_t2).  Outputs in the reference's order:
// mass, normal/t1/t2 momentum, energy, B_t1, B_t2 fluxes.
//
// The reference's double literals (0.5*, 2.0*, 1.0/) promote some
// sub-expressions to double; those are evaluated in double here too.  Where
// the promotion wraps a single float division or square root of float
// operands the double-rounded result equals the float result (53 >= 2*24+2),
// and the float form is used.
struct HlldIn {
  float dl, dr, ul, ur, vl, vr, wl, wr, pl, pr, byl, byr, bzl, bzr;
};

__host__ __device__ __forceinline__ void hlld_flux(const float gamma, const float Bx, const HlldIn &s,
                                          float f[7]) {
  const float TINY = 1.0e-10f;
  const float dens_L = s.dl, dens_R = s.dr, velx_L = s.ul, velx_R = s.ur;
  const float vely_L = s.vl, vely_R = s.vr, velz_L = s.wl, velz_R = s.wr;
  const float pres_L = s.pl, pres_R = s.pr, By_L = s.byl, By_R = s.byr;
  const float Bz_L = s.bzl, Bz_R = s.bzr;


  const float momx_L = dens_L * velx_L, momy_L = dens_L * vely_L, momz_L = dens_L * velz_L;
  const float momx_R = dens_R * velx_R, momy_R = dens_R * vely_R, momz_R = dens_R * velz_R;

  const float B2x = Bx * Bx;
  const float B2_L = B2x + By_L * By_L + Bz_L * Bz_L;
  const float v2_L = velx_L * velx_L + vely_L * vely_L + velz_L * velz_L;
  const float B2_R = B2x + By_R * By_R + Bz_R * Bz_R;
  const float v2_R = velx_R * velx_R + vely_R * vely_R + velz_R * velz_R;
  const float gm1 = gamma - 1.0f;
#if NMHD_FAST_ARITH
  const float etot_L = pres_L / gm1 + 0.5f * dens_L * v2_L + 0.5f * B2_L;
  const float etot_R = pres_R / gm1 + 0.5f * dens_R * v2_R + 0.5f * B2_R;
#else
  // etot = p/(gamma-1) + 0.5*rho*v2 + 0.5*B2, the last two terms in double
  const float etot_L = (float)((double)(pres_L / gm1) + 0.5 * (double)dens_L * (double)v2_L +
                               0.5 * (double)B2_L);
  const float etot_R = (float)((double)(pres_R / gm1) + 0.5 * (double)dens_R * (double)v2_R +
                               0.5 * (double)B2_R);
#endif

  const float gpl = gamma * pres_L, gpr = gamma * pres_R;
  const float gpbl = gpl + B2_L, gpbr = gpr + B2_R;
  const float fsig = 1.41421354f;  // sqrtf(2.0f)
  // sqrt((gpb + sqrt(gpb^2 - 4 gp Bx^2)) / (2.0*rho)): a float quotient
  const float cfl = sqrtf((gpbl + sqrtf(gpbl * gpbl - 4.0f * gpl * B2x)) / (2.0f * dens_L));
  const float cfr = sqrtf((gpbr + sqrtf(gpbr * gpbr - 4.0f * gpr * B2x)) / (2.0f * dens_R));
  const float cfmax = fsig * fmaxf(cfl, cfr);
  const float S_L = fminf(velx_L, velx_R) - cfmax;
  const float S_R = fmaxf(velx_L, velx_R) + cfmax;

#if NMHD_FAST_ARITH
  const float pT_L = pres_L + 0.5f * B2_L;
  const float pT_R = pres_R + 0.5f * B2_R;
  const float sRv = S_R - velx_R, sLv = S_L - velx_L;
  const float rden = 1.0f / (sRv * dens_R - sLv * dens_L);
  const float S_M = (sRv * momx_R - sLv * momx_L - pT_R + pT_L) * rden;
  const float pT_s = (sRv * dens_R * pT_L - sLv * dens_L * pT_R + dens_L * dens_R * sRv * sLv * (velx_R - velx_L)) * rden;
#else
  // p + 0.5*B2: exact 0.5*B2 in double, one double add, rounded to float
  const float pT_L = (float)((double)pres_L + 0.5 * (double)B2_L);
  const float pT_R = (float)((double)pres_R + 0.5 * (double)B2_R);

  const float sRv = S_R - velx_R, sLv = S_L - velx_L;
  const float den = sRv * dens_R - sLv * dens_L;
  const double rden = 1.0 / (double)den;
  float S_M = sRv * momx_R - sLv * momx_L - pT_R + pT_L;
  S_M = (float)((double)S_M * rden);
  float pT_s = sRv * dens_R * pT_L - sLv * dens_L * pT_R;
  pT_s = pT_s + dens_L * dens_R * sRv * sLv * (velx_R - velx_L);
  pT_s = (float)((double)pT_s * rden);
#endif

  const float sLm = S_L - S_M, sRm = S_R - S_M;
  // Single-star densities of both sides fix the Alfven speeds S_L*, S_R*
  // and with them the fan region; everything else of the star states is
  // computed below only for the side(s) the region's formula reads.
  const float dsL = dens_L * sLv;
  const float dsR = dens_R * sRv;
  const float dens_L_s = dsL / sLm;
  const float dens_R_s = dsR / sRm;
  const float sdL = sqrtf(dens_L_s), sdR = sqrtf(dens_R_s);
  const float S_L_s = S_M - fabsf(Bx) / sdL;
  const float S_R_s = S_M + fabsf(Bx) / sdR;

  // Region of the fan that contains x/t = 0.
  int region;
  if (S_L > 0.0f) region = 0;
  else if (S_L <= 0.0f && 0.0f <= S_L_s) region = 1;
  else if (S_L_s <= 0.0f && 0.0f <= S_M) region = 2;
  else if (S_M <= 0.0f && 0.0f <= S_R_s) region = 3;
  else if (S_R_s <= 0.0f && 0.0f <= S_R) region = 4;
  else region = 5;

  const bool left = region <= 2;
  // Side-selected quantities: every region formula uses one side only.
  const float d_ = left ? dens_L : dens_R;
  const float u_ = left ? velx_L : velx_R;
  const float v_ = left ? vely_L : vely_R;
  const float w_ = left ? velz_L : velz_R;
  const float by_ = left ? By_L : By_R;
  const float bz_ = left ? Bz_L : Bz_R;
  const float e_ = left ? etot_L : etot_R;
  const float pT_ = left ? pT_L : pT_R;
  const float mx_ = left ? momx_L : momx_R;
  const float my_ = left ? momy_L : momy_R;
  const float mz_ = left ? momz_L : momz_R;
  const float vB_ = u_ * Bx + v_ * by_ + w_ * bz_;

  const float F0 = d_ * u_;
  const float F1 = mx_ * u_ + pT_ - B2x;
  const float F2 = my_ * u_ - Bx * by_;
  const float F3 = mz_ * u_ - Bx * bz_;
  const float F4 = e_ * u_ + pT_ * u_ - Bx * vB_;
  const float F5 = by_ * u_ - Bx * v_;
  const float F6 = bz_ * u_ - Bx * w_;
  if (region == 0 || region == 5) {
    f[0] = F0; f[1] = F1; f[2] = F2; f[3] = F3; f[4] = F4; f[5] = F5; f[6] = F6;
    return;
  }
  // single-star state of the selected side (hlld.inl:146-164, the same
  // expressions for L and R)
  const float S_ = left ? S_L : S_R;
  const float sv_ = left ? sLv : sRv;
  const float sm_ = left ? sLm : sRm;
  const float ds_ = left ? dens_L_s : dens_R_s;
  const float dn_ = (left ? dsL : dsR) * sm_ - B2x + TINY;
  const float vs_ = v_ - Bx * by_ * (S_M - u_) / dn_;
  const float ws_ = w_ - Bx * bz_ * (S_M - u_) / dn_;
  const float q_ = d_ * (sv_ * sv_) - B2x;
  const float bys_ = by_ * q_ / dn_;
  const float bzs_ = bz_ * q_ / dn_;
  const float vBs_ = S_M * Bx + vs_ * bys_ + ws_ * bzs_;
  const float es_ = (sv_ * e_ - pT_ * u_ + pT_s * S_M + Bx * (vB_ - vBs_)) / sm_;
  // U* of the selected side
  const float Us1 = ds_ * S_M, Us2 = ds_ * vs_, Us3 = ds_ * ws_;
  if (region == 1 || region == 4) {
    f[0] = F0 + S_ * ds_ - S_ * d_;
    f[1] = F1 + S_ * Us1 - S_ * mx_;
    f[2] = F2 + S_ * Us2 - S_ * my_;
    f[3] = F3 + S_ * Us3 - S_ * mz_;
    f[4] = F4 + S_ * es_ - S_ * e_;
    f[5] = F5 + S_ * bys_ - S_ * by_;
    f[6] = F6 + S_ * bzs_ - S_ * bz_;
    return;
  }
  // regions 2 and 3: the other side's transverse star state too
  const float uo = left ? velx_R : velx_L;
  const float dno = (left ? dsR : dsL) * (left ? sRm : sLm) - B2x + TINY;
  const float svo = left ? sRv : sLv;
  const float qo = (left ? dens_R : dens_L) * (svo * svo) - B2x;
  const float byo = left ? By_R : By_L, bzo = left ? Bz_R : Bz_L;
  const float vso = (left ? vely_R : vely_L) - Bx * byo * (S_M - uo) / dno;
  const float wso = (left ? velz_R : velz_L) - Bx * bzo * (S_M - uo) / dno;
  const float byso = byo * qo / dno;
  const float bzso = bzo * qo / dno;
  const float vely_L_s = left ? vs_ : vso, vely_R_s = left ? vso : vs_;
  const float velz_L_s = left ? ws_ : wso, velz_R_s = left ? wso : ws_;
  const float By_L_s = left ? bys_ : byso, By_R_s = left ? byso : bys_;
  const float Bz_L_s = left ? bzs_ : bzso, Bz_R_s = left ? bzso : bzs_;
  // sign(Bx) as the reference computes it, Bx / |Bx| for |Bx| > 0, else 0:
  // the quotient is exactly +-1 for finite Bx and NaN for infinite Bx, so it
  // is written without the division
  float signBx = 0.0f;
  if (fabsf(Bx) > 0.0f) signBx = isinf(Bx) ? __builtin_nanf("") : copysignf(1.0f, Bx);
  // double-star states (hlld.inl:172-193)
  const float fr = 1.0f / (sdL + sdR);
  const float vely_ss = fr * (sdL * vely_L_s + sdR * vely_R_s + (By_R_s - By_L_s) * signBx);
  const float velz_ss = fr * (sdL * velz_L_s + sdR * velz_R_s + (Bz_R_s - Bz_L_s) * signBx);
  const float sdLR = sqrtf(dens_L_s * dens_R_s);
  const float By_ss = fr * (sdL * By_R_s + sdR * By_L_s + sdLR * (vely_R_s - vely_L_s) * signBx);
  const float Bz_ss = fr * (sdL * Bz_R_s + sdR * Bz_L_s + sdLR * (velz_R_s - velz_L_s) * signBx);
  const float vB_ss = S_M * Bx + vely_ss * By_ss + velz_ss * Bz_ss;
  const float Sss = left ? S_L_s : S_R_s;
  const float ess = left ? (es_ - sdL * (vBs_ - vB_ss) * signBx) : (es_ + sdR * (vBs_ - vB_ss) * signBx);
  const float Sd = Sss - S_;
  f[0] = F0 + Sss * ds_ - Sd * ds_ - S_ * d_;
  f[1] = F1 + Sss * Us1 - Sd * Us1 - S_ * mx_;
  f[2] = F2 + Sss * (ds_ * vely_ss) - Sd * Us2 - S_ * my_;
  f[3] = F3 + Sss * (ds_ * velz_ss) - Sd * Us3 - S_ * mz_;
  f[4] = F4 + Sss * ess - Sd * es_ - S_ * e_;
  f[5] = F5 + Sss * By_ss - Sd * bys_ - S_ * by_;
  f[6] = F6 + Sss * Bz_ss - Sd * bzs_ - S_ * bz_;
}

}  // namespace nmhd
