// HLLD flux over a generic scalar type, and its hand-written adjoint.
//
// hlld_tape() evaluates src/library/hlld.inl:7-284 (the `#if 1` fast
// magnetosonic bounds) keeping every intermediate; it is operation for
// operation the production hlld_flux() of mhd_math.cuh, including the
// reference's double-literal promotions (done in Traits<T>::wide), so with
// T = float it reproduces the production flux and its fan region bit for bit,
// and with T = double the reference's Real = double build.
//
// hlld_adjoint() is reverse-mode differentiation of that evaluation with the
// fan region, the min/max choices and sign(Bx) frozen at the values taken:
// given the adjoint of the 7 fluxes it returns the adjoint of the 14 left /
// right states and of the normal field.  The derivation is written out step by
// step below; every forward intermediate is read from the tape.
#pragma once
#include "ad_scalar.cuh"

namespace nmhd {
namespace ad {

// Left/right Riemann states: rho, v_n, v_t1, v_t2, p, B_t1, B_t2.
template <class T>
struct HState {
  T dl, dr, ul, ur, vl, vr, wl, wr, pl, pr, byl, byr, bzl, bzr;
};

// Per-side intermediates (names follow hlld.inl with the side suffix dropped).
template <class T>
struct HSide {
  T d, u, v, w, p, by, bz;                           // state
  T mx, my, mz, B2, v2, e, gp, gpb, disc, sq, num, cf, pT;
  T sv, sm, ds, dn, vs, ws, q, bys, bzs, vB, vBs, es, sd, Ss;
};

template <class T>
struct HTape {
  HSide<T> L, R;
  T Bx, B2x, absBx, sgn, cfmax, S_L, S_R, den, SMn, S_M, pTn, pT_s;
  T fr, vss, wss, sdLR, Byss, Bzss, vBss, eLss, eRss;
  int region;
};

template <class T>
NMHD_HD void hlld_side_pre(const T gamma, const T gm1, const T Bx, const T B2x, HSide<T> &s) {
  typedef typename Traits<T>::wide W;
  s.mx = s.d * s.u;
  s.my = s.d * s.v;
  s.mz = s.d * s.w;
  s.B2 = B2x + s.by * s.by + s.bz * s.bz;
  s.v2 = s.u * s.u + s.v * s.v + s.w * s.w;
  // etot = p/(gamma-1) + 0.5*rho*v2 + 0.5*B2, the last two terms in double
  s.e = to<T>(to<W>(s.p / gm1) + W(0.5) * to<W>(s.d) * to<W>(s.v2) + W(0.5) * to<W>(s.B2));
  s.gp = gamma * s.p;
  s.gpb = s.gp + s.B2;
  s.disc = s.gpb * s.gpb - T(4.0f) * s.gp * B2x;
  s.sq = gsqrt(s.disc);
  s.num = s.gpb + s.sq;
  s.cf = gsqrt(s.num / (T(2.0f) * s.d));
  s.pT = to<T>(to<W>(s.p) + W(0.5) * to<W>(s.B2));
  (void)Bx;
}

// Star state of one side; S = S_L or S_R, sign = -1 (left) or +1 (right).
template <class T>
NMHD_HD void hlld_side_star(const T Bx, const T B2x, const T TINY, const T S, const T S_M, HSide<T> &s) {
  s.sm = S - S_M;
  s.ds = s.d * s.sv / s.sm;
  s.dn = s.d * s.sv * s.sm - B2x + TINY;
  s.vs = s.v - Bx * s.by * (S_M - s.u) / s.dn;
  s.ws = s.w - Bx * s.bz * (S_M - s.u) / s.dn;
  s.q = s.d * (s.sv * s.sv) - B2x;
  s.bys = s.by * s.q / s.dn;
  s.bzs = s.bz * s.q / s.dn;
}

template <class T>
NMHD_HD void hlld_side_energy(const T Bx, const T S_M, const T pT_s, HSide<T> &s) {
  s.vB = s.u * Bx + s.v * s.by + s.w * s.bz;
  s.vBs = S_M * Bx + s.vs * s.bys + s.ws * s.bzs;
  s.es = (s.sv * s.e - s.pT * s.u + pT_s * S_M + Bx * (s.vB - s.vBs)) / s.sm;
  s.sd = gsqrt(s.ds);
}

template <class T>
NMHD_HD void hlld_tape(const T gamma, const T Bx, const HState<T> &in, HTape<T> &t) {
  typedef typename Traits<T>::wide W;
  typedef typename Traits<T>::real R;
  const T TINY = to<T>((R)1.0e-10);
  t.Bx = Bx;
  const R bxv = val(Bx);
  t.sgn = to<T>(bxv > R(0) ? R(1) : (bxv < R(0) ? R(-1) : R(0)));
  t.absBx = gabs(Bx);
  t.L.d = in.dl; t.L.u = in.ul; t.L.v = in.vl; t.L.w = in.wl; t.L.p = in.pl; t.L.by = in.byl; t.L.bz = in.bzl;
  t.R.d = in.dr; t.R.u = in.ur; t.R.v = in.vr; t.R.w = in.wr; t.R.p = in.pr; t.R.by = in.byr; t.R.bz = in.bzr;
  t.B2x = Bx * Bx;
  const T gm1 = gamma - T(1.0f);
  hlld_side_pre(gamma, gm1, Bx, t.B2x, t.L);
  hlld_side_pre(gamma, gm1, Bx, t.B2x, t.R);
  const T fsig = to<T>(1.41421354f);  // (float)sqrt(2.0) in both reference builds
  t.cfmax = fsig * gmax(t.L.cf, t.R.cf);
  t.S_L = gmin(t.L.u, t.R.u) - t.cfmax;
  t.S_R = gmax(t.L.u, t.R.u) + t.cfmax;
  t.R.sv = t.S_R - t.R.u;
  t.L.sv = t.S_L - t.L.u;
  t.den = t.R.sv * t.R.d - t.L.sv * t.L.d;
  const W rden = W(1.0) / to<W>(t.den);
  t.SMn = t.R.sv * t.R.mx - t.L.sv * t.L.mx - t.R.pT + t.L.pT;
  t.S_M = to<T>(to<W>(t.SMn) * rden);
  t.pTn = t.R.sv * t.R.d * t.L.pT - t.L.sv * t.L.d * t.R.pT;
  t.pTn = t.pTn + t.L.d * t.R.d * t.R.sv * t.L.sv * (t.R.u - t.L.u);
  t.pT_s = to<T>(to<W>(t.pTn) * rden);
  hlld_side_star(Bx, t.B2x, TINY, t.S_L, t.S_M, t.L);
  hlld_side_star(Bx, t.B2x, TINY, t.S_R, t.S_M, t.R);
  hlld_side_energy(Bx, t.S_M, t.pT_s, t.L);
  hlld_side_energy(Bx, t.S_M, t.pT_s, t.R);
  t.L.Ss = t.S_M - t.absBx / t.L.sd;
  t.R.Ss = t.S_M + t.absBx / t.R.sd;
  const R SL = val(t.S_L), SLs = val(t.L.Ss), SM = val(t.S_M), SRs = val(t.R.Ss), SR = val(t.S_R);
  int region;
  if (SL > R(0)) region = 0;
  else if (SL <= R(0) && R(0) <= SLs) region = 1;
  else if (SLs <= R(0) && R(0) <= SM) region = 2;
  else if (SM <= R(0) && R(0) <= SRs) region = 3;
  else if (SRs <= R(0) && R(0) <= SR) region = 4;
  else region = 5;
  t.region = region;
  if (region == 2 || region == 3) {
    const T sgn = t.sgn;
    t.fr = T(1.0f) / (t.L.sd + t.R.sd);
    t.vss = t.fr * (t.L.sd * t.L.vs + t.R.sd * t.R.vs + (t.R.bys - t.L.bys) * sgn);
    t.wss = t.fr * (t.L.sd * t.L.ws + t.R.sd * t.R.ws + (t.R.bzs - t.L.bzs) * sgn);
    t.sdLR = gsqrt(t.L.ds * t.R.ds);
    t.Byss = t.fr * (t.L.sd * t.R.bys + t.R.sd * t.L.bys + t.sdLR * (t.R.vs - t.L.vs) * sgn);
    t.Bzss = t.fr * (t.L.sd * t.R.bzs + t.R.sd * t.L.bzs + t.sdLR * (t.R.ws - t.L.ws) * sgn);
    t.vBss = t.S_M * Bx + t.vss * t.Byss + t.wss * t.Bzss;
    t.eLss = t.L.es - t.L.sd * (t.L.vBs - t.vBss) * sgn;
    t.eRss = t.R.es + t.R.sd * (t.R.vBs - t.vBss) * sgn;
  }
}

// The flux of the region on the tape (hlld.inl:229-284); kLeft selects the
// side at compile time (regions 0-2 use the left state, 3-5 the right).
template <bool kLeft, class T>
NMHD_HD void hlld_flux_side(const HTape<T> &t, T f[7]) {
  const HSide<T> &s = kLeft ? t.L : t.R;
  const T Bx = t.Bx;
  const T F0 = s.d * s.u;
  const T F1 = s.mx * s.u + s.pT - t.B2x;
  const T F2 = s.my * s.u - Bx * s.by;
  const T F3 = s.mz * s.u - Bx * s.bz;
  const T F4 = s.e * s.u + s.pT * s.u - Bx * s.vB;
  const T F5 = s.by * s.u - Bx * s.v;
  const T F6 = s.bz * s.u - Bx * s.w;
  if (t.region == 0 || t.region == 5) {
    f[0] = F0; f[1] = F1; f[2] = F2; f[3] = F3; f[4] = F4; f[5] = F5; f[6] = F6;
    return;
  }
  const T S = kLeft ? t.S_L : t.S_R;
  const T Us1 = s.ds * t.S_M, Us2 = s.ds * s.vs, Us3 = s.ds * s.ws;
  if (t.region == 1 || t.region == 4) {
    f[0] = F0 + S * s.ds - S * s.d;
    f[1] = F1 + S * Us1 - S * s.mx;
    f[2] = F2 + S * Us2 - S * s.my;
    f[3] = F3 + S * Us3 - S * s.mz;
    f[4] = F4 + S * s.es - S * s.e;
    f[5] = F5 + S * s.bys - S * s.by;
    f[6] = F6 + S * s.bzs - S * s.bz;
    return;
  }
  const T Sss = s.Ss;
  const T ess = kLeft ? t.eLss : t.eRss;
  const T Sd = Sss - S;
  f[0] = F0 + Sss * s.ds - Sd * s.ds - S * s.d;
  f[1] = F1 + Sss * Us1 - Sd * Us1 - S * s.mx;
  f[2] = F2 + Sss * (s.ds * t.vss) - Sd * Us2 - S * s.my;
  f[3] = F3 + Sss * (s.ds * t.wss) - Sd * Us3 - S * s.mz;
  f[4] = F4 + Sss * ess - Sd * s.es - S * s.e;
  f[5] = F5 + Sss * t.Byss - Sd * s.bys - S * s.by;
  f[6] = F6 + Sss * t.Bzss - Sd * s.bzs - S * s.bz;
}

template <class T>
NMHD_HD void hlld_flux_of(const HTape<T> &t, T f[7]) {
  if (t.region <= 2) hlld_flux_side<true>(t, f);
  else hlld_flux_side<false>(t, f);
}

template <class T>
NMHD_HD void hlld_g(const T gamma, const T Bx, const HState<T> &in, T f[7]) {
  HTape<T> t;
  hlld_tape(gamma, Bx, in, t);
  hlld_flux_of(t, f);
}

// ---------------------------------------------------------------------------
// Adjoint.  A<R> holds the adjoints of one side's intermediates.
template <class R>
struct HAdj {
  R d, u, v, w, p, by, bz, mx, my, mz, B2, v2, e, pT, vB, sv, sm, ds, dn, vs, ws, q, bys, bzs, vBs, es, sd, cf;
};

template <class R>
NMHD_HD void hadj_zero(HAdj<R> &a) {
  a.d = a.u = a.v = a.w = a.p = a.by = a.bz = a.mx = a.my = a.mz = R(0);
  a.B2 = a.v2 = a.e = a.pT = a.vB = a.sv = a.sm = a.ds = a.dn = a.vs = a.ws = R(0);
  a.q = a.bys = a.bzs = a.vBs = a.es = a.sd = a.cf = R(0);
}

// Reverse of hlld_side_energy and hlld_side_star for one side.  The reverse
// sweep needs no correctly rounded quotients: each denominator is inverted
// once and multiplied (the forward tape above keeps the exact divisions).
template <class R>
NMHD_HD void hlld_side_star_rev(const HSide<R> &s, const R Bx, const R S_M, const R pT_s, HAdj<R> &a, R &aSM,
                                R &apTs, R &aBx, R &aB2x, R &aS) {
  const R ism = R(1) / s.sm, idn = R(1) / s.dn;
  // sd = sqrt(ds)
  if (s.sd > R(0)) a.ds += a.sd * (R(0.5) / s.sd);
  // es = (sv*e - pT*u + pT_s*S_M + Bx*(vB - vBs)) / sm
  {
    const R t = a.es * ism;
    a.sv = fmaa(t, s.e, a.sv);
    a.e = fmaa(t, s.sv, a.e);
    a.pT = fmaa(-t, s.u, a.pT);
    a.u = fmaa(-t, s.pT, a.u);
    apTs = fmaa(t, S_M, apTs);
    aSM = fmaa(t, pT_s, aSM);
    aBx = fmaa(t, (s.vB - s.vBs), aBx);
    a.vB = fmaa(t, Bx, a.vB);
    a.vBs = fmaa(-t, Bx, a.vBs);
    a.sm = fmaa(-t, s.es, a.sm);
  }
  // vBs = S_M*Bx + vs*bys + ws*bzs
  aSM = fmaa(a.vBs, Bx, aSM);
  aBx = fmaa(a.vBs, S_M, aBx);
  a.vs = fmaa(a.vBs, s.bys, a.vs);
  a.bys = fmaa(a.vBs, s.vs, a.bys);
  a.ws = fmaa(a.vBs, s.bzs, a.ws);
  a.bzs = fmaa(a.vBs, s.ws, a.bzs);
  // bys = by*q/dn, bzs = bz*q/dn
  a.by = fmaa(a.bys * s.q, idn, a.by);
  a.bz = fmaa(a.bzs * s.q, idn, a.bz);
  a.q = fmaa((a.bys * s.by + a.bzs * s.bz), idn, a.q);
  a.dn = fmaa(-(a.bys * s.bys + a.bzs * s.bzs), idn, a.dn);
  // q = d*sv^2 - B2x
  a.d = fmaa(a.q * s.sv, s.sv, a.d);
  a.sv = fmaa(a.q * R(2) * s.d, s.sv, a.sv);
  aB2x -= a.q;
  // vs = v - Bx*by*(S_M - u)/dn, ws = w - Bx*bz*(S_M - u)/dn
  {
    const R g = (S_M - s.u) * idn;
    const R tv = -a.vs, tw = -a.ws;
    a.v += a.vs;
    a.w += a.ws;
    aBx = fmaa((tv * s.by + tw * s.bz), g, aBx);
    a.by = fmaa(tv * Bx, g, a.by);
    a.bz = fmaa(tw * Bx, g, a.bz);
    const R c = (tv * s.by + tw * s.bz) * Bx * idn;
    aSM += c;
    a.u -= c;
    a.dn = fmaa(-c, g, a.dn);
  }
  // dn = d*sv*sm - B2x + TINY
  a.d = fmaa(a.dn * s.sv, s.sm, a.d);
  a.sv = fmaa(a.dn * s.d, s.sm, a.sv);
  a.sm = fmaa(a.dn * s.d, s.sv, a.sm);
  aB2x -= a.dn;
  // ds = d*sv/sm
  {
    const R t = a.ds * ism;
    a.d = fmaa(t, s.sv, a.d);
    a.sv = fmaa(t, s.d, a.sv);
    a.sm = fmaa(-t, s.ds, a.sm);
  }
  // sm = S - S_M
  aS += a.sm;
  aSM -= a.sm;
}

// Reverse of vB = u*Bx + v*by + w*bz (used by the flux of every region).
template <class R>
NMHD_HD void hlld_side_vB_rev(const HSide<R> &s, const R Bx, HAdj<R> &a, R &aBx) {
  a.u = fmaa(a.vB, Bx, a.u);
  aBx = fmaa(a.vB, s.u, aBx);
  a.v = fmaa(a.vB, s.by, a.v);
  a.by = fmaa(a.vB, s.v, a.by);
  a.w = fmaa(a.vB, s.bz, a.w);
  a.bz = fmaa(a.vB, s.w, a.bz);
}

// Reverse of hlld_side_pre (after pT, cf, e, mx.. have their adjoints).
template <class R>
NMHD_HD void hlld_side_pre_rev(const HSide<R> &s, const R gamma, const R igm1, const R B2x, HAdj<R> &a,
                               R &aB2x) {
  // pT = p + 0.5*B2
  a.p += a.pT;
  a.B2 = fmaa(R(0.5), a.pT, a.B2);
  // cf = sqrt(num/(2d))
  if (s.cf > R(0)) {
    const R id = R(1) / s.d;
    const R aQ = a.cf * (R(0.5) / s.cf);
    const R Q = R(0.5) * s.num * id;
    const R anum = R(0.5) * aQ * id;
    a.d = fmaa(-(aQ * Q), id, a.d);
    // num = gpb + sq; sq = sqrt(disc); disc = gpb^2 - 4 gp B2x; gpb = gp + B2
    R agpb = anum, agp = R(0);
    if (s.sq > R(0)) {
      const R adisc = anum * (R(0.5) / s.sq);
      agpb = fmaa(adisc * R(2), s.gpb, agpb);
      agp = fmaa(-(adisc * R(4)), B2x, agp);
      aB2x = fmaa(-(adisc * R(4)), s.gp, aB2x);
    }
    agp += agpb;
    a.B2 += agpb;
    a.p = fmaa(gamma, agp, a.p);
  }
  // e = p/gm1 + 0.5*d*v2 + 0.5*B2
  a.p = fmaa(a.e, igm1, a.p);
  a.d = fmaa(R(0.5) * a.e, s.v2, a.d);
  a.v2 = fmaa(R(0.5) * a.e, s.d, a.v2);
  a.B2 = fmaa(R(0.5), a.e, a.B2);
  // v2, B2, momenta
  a.u = fmaa(R(2) * s.u, a.v2, a.u);
  a.v = fmaa(R(2) * s.v, a.v2, a.v);
  a.w = fmaa(R(2) * s.w, a.v2, a.w);
  aB2x += a.B2;
  a.by = fmaa(R(2) * s.by, a.B2, a.by);
  a.bz = fmaa(R(2) * s.bz, a.B2, a.bz);
  a.d = fmaa(a.mz, s.w, fmaa(a.my, s.v, fmaa(a.mx, s.u, a.d)));
  a.u = fmaa(a.mx, s.d, a.u);
  a.v = fmaa(a.my, s.d, a.v);
  a.w = fmaa(a.mz, s.d, a.w);
}


// Reverse of the region flux (hlld_flux_side) and of the double-star states.
// The fan side (left for regions 0-2, right for 3-5) is data, not control
// flow: the side's quantities are selected, the adjoints accumulated in aX and
// handed to its side at the end, and the sign sx = -1 (left) / +1 (right)
// carries the two sides' mirror formulas (S_L* = S_M - |Bx|/sdL vs S_R* = S_M
// + |Bx|/sdR, eL** = eL* - sdL(...) vs eR** = eR* + sdR(...)).  Faces of one
// warp with fan regions on both sides then take one path.
template <class R>
NMHD_HD void hlld_region_rev(const HTape<R> &t, const R lf[7], HAdj<R> &aL, HAdj<R> &aR, R &aBx, R &aB2x,
                             R &aSM, R &aSL, R &aSR, R &aabs) {
  const int rg = t.region;
  const bool left = rg <= 2;
  const R sx = left ? R(-1) : R(1);
  // the side's forward quantities
  const R d = left ? t.L.d : t.R.d, u = left ? t.L.u : t.R.u, v = left ? t.L.v : t.R.v;
  const R w = left ? t.L.w : t.R.w, by = left ? t.L.by : t.R.by, bz = left ? t.L.bz : t.R.bz;
  const R mx = left ? t.L.mx : t.R.mx, my = left ? t.L.my : t.R.my, mz = left ? t.L.mz : t.R.mz;
  const R e = left ? t.L.e : t.R.e, pT = left ? t.L.pT : t.R.pT, vB = left ? t.L.vB : t.R.vB;
  const R Bx = t.Bx, sgn = t.sgn;
  HAdj<R> aX;
  hadj_zero(aX);
  R aSX = R(0);
  // F = F(U) of side X
  aX.d = fmaa(lf[0], u, aX.d);
  aX.u = fmaa(lf[6], bz, fmaa(lf[5], by, fmaa(lf[4], (e + pT), fmaa(lf[3], mz, fmaa(lf[2], my, fmaa(lf[1], mx, fmaa(lf[0], d, aX.u)))))));
  aX.mx = fmaa(lf[1], u, aX.mx);
  aX.pT = fmaa(lf[4], u, aX.pT + lf[1]);
  aB2x -= lf[1];
  aX.my = fmaa(lf[2], u, aX.my);
  aX.mz = fmaa(lf[3], u, aX.mz);
  aBx = fmaa(-lf[6], w, fmaa(-lf[5], v, fmaa(-lf[4], vB, fmaa(-lf[3], bz, fmaa(-lf[2], by, aBx)))));
  aX.by = fmaa(-lf[2], Bx, fmaa(lf[5], u, aX.by));
  aX.bz = fmaa(-lf[3], Bx, fmaa(lf[6], u, aX.bz));
  aX.e = fmaa(lf[4], u, aX.e);
  aX.vB = fmaa(-lf[4], Bx, aX.vB);
  aX.v = fmaa(-lf[5], Bx, aX.v);
  aX.w = fmaa(-lf[6], Bx, aX.w);
  if (rg != 0 && rg != 5) {
    const R S = left ? t.S_L : t.S_R;
    const R ds = left ? t.L.ds : t.R.ds, vs = left ? t.L.vs : t.R.vs, ws = left ? t.L.ws : t.R.ws;
    const R es = left ? t.L.es : t.R.es, bys = left ? t.L.bys : t.R.bys, bzs = left ? t.L.bzs : t.R.bzs;
    const R Us1 = ds * t.S_M, Us2 = ds * vs, Us3 = ds * ws;
    // -S*U
    aX.d = fmaa(-S, lf[0], aX.d);
    aX.mx = fmaa(-S, lf[1], aX.mx);
    aX.my = fmaa(-S, lf[2], aX.my);
    aX.mz = fmaa(-S, lf[3], aX.mz);
    aX.e = fmaa(-S, lf[4], aX.e);
    aX.by = fmaa(-S, lf[5], aX.by);
    aX.bz = fmaa(-S, lf[6], aX.bz);
    // d/dS of S*(U* - U) (regions 1, 4) and of -(Sss - S)*U* - S*U (regions 2, 3)
    aSX = fmaa(lf[6], (bzs - bz), fmaa(lf[5], (bys - by), fmaa(lf[4], (es - e), fmaa(lf[3], (Us3 - mz), fmaa(lf[2], (Us2 - my), fmaa(lf[1], (Us1 - mx), fmaa(lf[0], (ds - d), aSX)))))));
    R cs = S;  // coefficient of U*
    const bool dstar = rg == 2 || rg == 3;
    if (dstar) {
      const R sd = left ? t.L.sd : t.R.sd, vBs = left ? t.L.vBs : t.R.vBs;
      const R Sss = left ? t.L.Ss : t.R.Ss;
      const R ess = left ? t.eLss : t.eRss;
      cs = -(Sss - S);
      const R aSss = lf[2] * (ds * t.vss - Us2) + lf[3] * (ds * t.wss - Us3) + lf[4] * (ess - es) +
                     lf[5] * (t.Byss - bys) + lf[6] * (t.Bzss - bzs);
      // Sss * U**
      aX.ds = fmaa(Sss, (lf[0] + lf[1] * t.S_M + lf[2] * t.vss + lf[3] * t.wss), aX.ds);
      aSM = fmaa(Sss * lf[1], ds, aSM);
      R avss = Sss * lf[2] * ds, awss = Sss * lf[3] * ds;
      const R aess = Sss * lf[4];
      R aByss = Sss * lf[5], aBzss = Sss * lf[6];
      // ess = eX* + sx * sdX * (vBX* - vBss) * sgn
      R avBss = R(0), afr = R(0), asdLR = R(0);
      aX.es += aess;
      aX.sd = fmaa(sx * aess * (vBs - t.vBss), sgn, aX.sd);
      aX.vBs = fmaa(sx * aess * sd, sgn, aX.vBs);
      avBss = fmaa(-(sx * aess * sd), sgn, avBss);
      // vBss = S_M*Bx + vss*Byss + wss*Bzss
      aSM = fmaa(avBss, Bx, aSM);
      aBx = fmaa(avBss, t.S_M, aBx);
      avss = fmaa(avBss, t.Byss, avss);
      aByss = fmaa(avBss, t.vss, aByss);
      awss = fmaa(avBss, t.Bzss, awss);
      aBzss = fmaa(avBss, t.wss, aBzss);
      // Bzss = fr*(sdL*bzRs + sdR*bzLs + sdLR*(wRs - wLs)*sgn)
      {
        const R n = t.L.sd * t.R.bzs + t.R.sd * t.L.bzs + t.sdLR * (t.R.ws - t.L.ws) * sgn;
        afr = fmaa(aBzss, n, afr);
        const R c = aBzss * t.fr;
        aL.sd = fmaa(c, t.R.bzs, aL.sd);
        aR.bzs = fmaa(c, t.L.sd, aR.bzs);
        aR.sd = fmaa(c, t.L.bzs, aR.sd);
        aL.bzs = fmaa(c, t.R.sd, aL.bzs);
        asdLR = fmaa(c * (t.R.ws - t.L.ws), sgn, asdLR);
        aR.ws = fmaa(c * t.sdLR, sgn, aR.ws);
        aL.ws = fmaa(-(c * t.sdLR), sgn, aL.ws);
      }
      // Byss = fr*(sdL*byRs + sdR*byLs + sdLR*(vRs - vLs)*sgn)
      {
        const R n = t.L.sd * t.R.bys + t.R.sd * t.L.bys + t.sdLR * (t.R.vs - t.L.vs) * sgn;
        afr = fmaa(aByss, n, afr);
        const R c = aByss * t.fr;
        aL.sd = fmaa(c, t.R.bys, aL.sd);
        aR.bys = fmaa(c, t.L.sd, aR.bys);
        aR.sd = fmaa(c, t.L.bys, aR.sd);
        aL.bys = fmaa(c, t.R.sd, aL.bys);
        asdLR = fmaa(c * (t.R.vs - t.L.vs), sgn, asdLR);
        aR.vs = fmaa(c * t.sdLR, sgn, aR.vs);
        aL.vs = fmaa(-(c * t.sdLR), sgn, aL.vs);
      }
      // wss = fr*(sdL*wLs + sdR*wRs + (bzRs - bzLs)*sgn)
      {
        const R n = t.L.sd * t.L.ws + t.R.sd * t.R.ws + (t.R.bzs - t.L.bzs) * sgn;
        afr = fmaa(awss, n, afr);
        const R c = awss * t.fr;
        aL.sd = fmaa(c, t.L.ws, aL.sd);
        aL.ws = fmaa(c, t.L.sd, aL.ws);
        aR.sd = fmaa(c, t.R.ws, aR.sd);
        aR.ws = fmaa(c, t.R.sd, aR.ws);
        aR.bzs = fmaa(c, sgn, aR.bzs);
        aL.bzs = fmaa(-c, sgn, aL.bzs);
      }
      // vss = fr*(sdL*vLs + sdR*vRs + (byRs - byLs)*sgn)
      {
        const R n = t.L.sd * t.L.vs + t.R.sd * t.R.vs + (t.R.bys - t.L.bys) * sgn;
        afr = fmaa(avss, n, afr);
        const R c = avss * t.fr;
        aL.sd = fmaa(c, t.L.vs, aL.sd);
        aL.vs = fmaa(c, t.L.sd, aL.vs);
        aR.sd = fmaa(c, t.R.vs, aR.sd);
        aR.vs = fmaa(c, t.R.sd, aR.vs);
        aR.bys = fmaa(c, sgn, aR.bys);
        aL.bys = fmaa(-c, sgn, aL.bys);
      }
      // sdLR = sqrt(dLs*dRs)
      if (t.sdLR > R(0)) {
        const R c = asdLR * (R(0.5) / t.sdLR);
        aL.ds = fmaa(c, t.R.ds, aL.ds);
        aR.ds = fmaa(c, t.L.ds, aR.ds);
      }
      // fr = 1/(sdL + sdR)
      {
        const R c = -afr * t.fr * t.fr;
        aL.sd += c;
        aR.sd += c;
      }
      // Sss = S_M + sx*|Bx|/sdX
      aSM += aSss;
      {
        const R isd = R(1) / sd;
        aabs = fmaa(sx * aSss, isd, aabs);
        aX.sd = fmaa(-(sx * aSss * t.absBx * isd), isd, aX.sd);
      }
    }
    aX.ds = fmaa(cs, (lf[0] + lf[1] * t.S_M + lf[2] * vs + lf[3] * ws), aX.ds);
    aSM = fmaa(cs * lf[1], ds, aSM);
    aX.vs = fmaa(cs * lf[2], ds, aX.vs);
    aX.ws = fmaa(cs * lf[3], ds, aX.ws);
    aX.es = fmaa(cs, lf[4], aX.es);
    aX.bys = fmaa(cs, lf[5], aX.bys);
    aX.bzs = fmaa(cs, lf[6], aX.bzs);
  }
  // hand the side-X adjoints to their side
  const R kl = left ? R(1) : R(0), kr = R(1) - kl;
#define NMHD_HAND(f) aL.f += kl * aX.f; aR.f += kr * aX.f;
  NMHD_HAND(d) NMHD_HAND(u) NMHD_HAND(v) NMHD_HAND(w) NMHD_HAND(by) NMHD_HAND(bz)
  NMHD_HAND(mx) NMHD_HAND(my) NMHD_HAND(mz) NMHD_HAND(e) NMHD_HAND(pT) NMHD_HAND(vB)
  NMHD_HAND(ds) NMHD_HAND(vs) NMHD_HAND(ws) NMHD_HAND(es) NMHD_HAND(bys) NMHD_HAND(bzs)
  NMHD_HAND(sd) NMHD_HAND(vBs)
#undef NMHD_HAND
  aSL = fmaa(kl, aSX, aSL);
  aSR = fmaa(kr, aSX, aSR);
}

// Adjoint of hlld_g: ls and lBx receive d<lf, f>/d(state) and d<lf, f>/dBx.
template <class R>
NMHD_HD void hlld_adjoint(const R gamma, const R Bx, const HState<R> &in, const R lf[7], HState<R> &ls,
                          R &lBx) {
  HTape<R> t;
  hlld_tape(gamma, Bx, in, t);
  const int rg = t.region;
  HAdj<R> aL, aR;
  hadj_zero(aL);
  hadj_zero(aR);
  R aBx = R(0), aB2x = R(0), aSM = R(0), apTs = R(0), aSL = R(0), aSR = R(0), aabs = R(0);
  const R sgn = t.sgn;
  hlld_region_rev(t, lf, aL, aR, aBx, aB2x, aSM, aSL, aSR, aabs);
  if (rg != 0 && rg != 5) {  // regions 0 and 5 use no wave speed or star state
    // --- star states of both sides ---------------------------------------------
    hlld_side_star_rev(t.L, Bx, t.S_M, t.pT_s, aL, aSM, apTs, aBx, aB2x, aSL);
    hlld_side_star_rev(t.R, Bx, t.S_M, t.pT_s, aR, aSM, apTs, aBx, aB2x, aSR);

    // --- S_M = SMn/den, pT* = pTn/den ---------------------------------------------
    {
      const R iden = R(1) / t.den;
      const R aSMn = aSM * iden, apTn = apTs * iden;
      const R aden = -(aSM * t.S_M + apTs * t.pT_s) * iden;
      const R dl = t.L.d, dr = t.R.d, sLv = t.L.sv, sRv = t.R.sv, du = t.R.u - t.L.u;
      // pTn = sRv*dr*pTL - sLv*dl*pTR + dl*dr*sRv*sLv*(ur - ul)
      aR.sv = fmaa(apTn, (dr * t.L.pT + dl * dr * sLv * du), aR.sv);
      aR.d = fmaa(apTn, (sRv * t.L.pT + dl * sRv * sLv * du), aR.d);
      aL.pT = fmaa(apTn * sRv, dr, aL.pT);
      aL.sv = fmaa(apTn, (-dl * t.R.pT + dl * dr * sRv * du), aL.sv);
      aL.d = fmaa(apTn, (-sLv * t.R.pT + dr * sRv * sLv * du), aL.d);
      aR.pT = fmaa(-(apTn * sLv), dl, aR.pT);
      aR.u = fmaa(apTn * dl * dr * sRv, sLv, aR.u);
      aL.u = fmaa(-(apTn * dl * dr * sRv), sLv, aL.u);
      // SMn = sRv*mxR - sLv*mxL - pTR + pTL
      aR.sv = fmaa(aSMn, t.R.mx, aR.sv);
      aR.mx = fmaa(aSMn, sRv, aR.mx);
      aL.sv = fmaa(-aSMn, t.L.mx, aL.sv);
      aL.mx = fmaa(-aSMn, sLv, aL.mx);
      aR.pT -= aSMn;
      aL.pT += aSMn;
      // den = sRv*dr - sLv*dl
      aR.sv = fmaa(aden, dr, aR.sv);
      aR.d = fmaa(aden, sRv, aR.d);
      aL.sv = fmaa(-aden, dl, aL.sv);
      aL.d = fmaa(-aden, sLv, aL.d);
    }
    // sv = S - u
    aSR += aR.sv;
    aR.u -= aR.sv;
    aSL += aL.sv;
    aL.u -= aL.sv;
    // S_L = min(uL, uR) - cfmax, S_R = max(uL, uR) + cfmax, cfmax = fsig*max(cfL, cfR)
    {
      if (t.R.u < t.L.u) aR.u += aSL; else aL.u += aSL;
      if (t.R.u > t.L.u) aR.u += aSR; else aL.u += aSR;
      const R acf = R(1.41421354f) * (aSR - aSL);
      if (t.R.cf > t.L.cf) aR.cf += acf; else aL.cf += acf;
    }
  }
  hlld_side_vB_rev(t.L, Bx, aL, aBx);
  hlld_side_vB_rev(t.R, Bx, aR, aBx);
  const R igm1 = R(1) / (gamma - R(1));
  hlld_side_pre_rev(t.L, gamma, igm1, t.B2x, aL, aB2x);
  hlld_side_pre_rev(t.R, gamma, igm1, t.B2x, aR, aB2x);
  aBx = fmaa(aabs, sgn, fmaa(R(2) * Bx, aB2x, aBx));

  ls.dl = aL.d; ls.dr = aR.d; ls.ul = aL.u; ls.ur = aR.u; ls.vl = aL.v; ls.vr = aR.v;
  ls.wl = aL.w; ls.wr = aR.w; ls.pl = aL.p; ls.pr = aR.p; ls.byl = aL.by; ls.byr = aR.by;
  ls.bzl = aL.bz; ls.bzr = aR.bz;
  lBx = aBx;
}

}  // namespace ad
}  // namespace nmhd
