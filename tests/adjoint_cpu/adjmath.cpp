// Host build of the device per-point math (bnz_device.cuh) and its VJPs
// (bnz_adjoint_math.h) for the CPU tests of the adjoint: the forward
// functions are evaluated here for finite differences, the VJPs are the ones
// the adjoint kernels call.  Test infrastructure only.
#include <cmath>

#define __device__
#define __forceinline__ inline
#include "../../bonzo_b200/csrc/bnz_device.cuh"
#include "../../bonzo_b200/csrc/bnz_adjoint_math.h"

extern "C" {

// forward Riemann flux (rs: 0 hll, 2 hlld, 3 hllt) of one face; wL[BX] is the normal field
void t_flux(int rs, const double* wL, const double* wR, double gam, double* f) {
  unsigned err = 0;
  double l[9], r[9];
  for (int n = 0; n < 9; ++n) {
    l[n] = wL[n];
    r[n] = wR[n];
  }
  r[dev::BX] = l[dev::BX];
  if (rs == 2) dev::flux_hlld(f, l, r, gam, err);
  else if (rs == 3) dev::flux_hllt(f, l, r, gam, err);
  else dev::flux_hll(f, l, r, gam);
}

void t_vjp_flux(int rs, const double* wL, const double* wR, double gam, const double* fb, double* wLb,
                double* wRb) {
  double l[9], r[9];
  for (int n = 0; n < 9; ++n) {
    l[n] = wL[n];
    r[n] = wR[n];
    wLb[n] = wRb[n] = 0.;
  }
  r[dev::BX] = l[dev::BX];
  if (rs == 2) adj::vjp_hlld(l, r, gam, fb, wLb, wRb);
  else if (rs == 3) adj::vjp_hllt(l, r, gam, fb, wLb, wRb);
  else adj::vjp_hll(l, r, gam, fb, wLb, wRb);
}

// HLLD wave-fan region (1..6) the forward selects for these states
int t_hlld_region(const double* wL, const double* wR, double gam) {
  double l[9], r[9];
  for (int n = 0; n < 9; ++n) {
    l[n] = wL[n];
    r[n] = wR[n];
  }
  r[dev::BX] = l[dev::BX];
  double sL, sR;
  dev::wave_speeds(l, r, gam, sL, sR);
  const double bx = l[dev::BX], bx2 = bx * bx;
  const double ptL = l[dev::PR] + 0.5 * (bx2 + l[dev::BY] * l[dev::BY] + l[dev::BZ] * l[dev::BZ]);
  const double ptR = r[dev::PR] + 0.5 * (bx2 + r[dev::BY] * r[dev::BY] + r[dev::BZ] * r[dev::BZ]);
  const double mxL = l[0] * l[1], mxR = r[0] * r[1];
  const double sM = (sR * mxR - sL * mxL - ((mxR * r[1] + ptR - bx2) - (mxL * l[1] + ptL - bx2))) /
                    (sR * r[0] - sL * l[0] - (mxR - mxL));
  const double rLs = l[0] * (sL - l[1]) / (sL - sM), rRs = r[0] * (sR - r[1]) / (sR - sM);
  const double sLs = sM - fabs(bx) / sqrt(rLs), sRs = sM + fabs(bx) / sqrt(rRs);
  int k = 0;
  if (sL > 0.) k = 1;
  if (sL <= 0. && 0. < sLs) k = 2;
  if (sLs <= 0. && 0. < sM) k = 3;
  if (sM <= 0. && 0. < sRs) k = 4;
  if (sRs <= 0. && 0. < sR) k = 5;
  if (sR <= 0.) k = 6;
  return k;
}

// HLLT wave-fan region (1..5, 0 where the forward flags ERR_FAN)
int t_hllt_region(const double* wL, const double* wR, double gam) {
  double l[9], r[9];
  for (int n = 0; n < 9; ++n) {
    l[n] = wL[n];
    r[n] = wR[n];
  }
  r[dev::BX] = l[dev::BX];
  double uL[9], uR[9], fL[9], fR[9];
  dev::prim2cons(uL, l, gam);
  dev::prim2cons(uR, r, gam);
  dev::primcons2flux(fL, l, uL);
  dev::primcons2flux(fR, r, uR);
  double sL, sR;
  dev::wave_speeds(l, r, gam, sL, sR);
  const double rhos = (sR * uR[0] - sL * uL[0] - (fR[0] - fL[0])) / (sR - sL);
  const double us = (sR * fL[0] - sL * fR[0] + sR * sL * (uR[0] - uL[0])) / (sR - sL) / rhos;
  const double a = fabs(l[dev::BX]) * sqrt(1. / rhos);
  const double sLs = us - a, sRs = us + a;
  int k = 0;
  if (sL > 0.) k = 1;
  if (sL <= 0. && 0. < sLs) k = 2;
  if (sLs <= 0. && 0. < sRs) k = 3;
  if (sRs <= 0. && 0. < sR) k = 4;
  if (sR <= 0.) k = 5;
  return k;
}

void t_cons2prim(const double* u, double gam, double* w) { dev::cons2prim(w, u, gam); }
void t_prim2cons(const double* w, double gam, double* u) { dev::prim2cons(u, w, gam); }
void t_vjp_cons2prim(const double* w, const double* wb, double gam, double* ub) {
  for (int n = 0; n < 9; ++n) ub[n] = 0.;
  adj::vjp_cons2prim(w, wb, gam, ub);
}
void t_vjp_prim2cons(const double* w, const double* ub, double gam, double* wb) {
  for (int n = 0; n < 9; ++n) wb[n] = 0.;
  adj::vjp_prim2cons(w, ub, gam, wb);
}

// PLM face states of one variable: out[0] = wL at face i, out[1] = wR
void t_plm(int lim, const double* c4, double* out) {
  double hl, hr;
  if (lim == 1) {
    hl = dev::half_slope<dev::LIM_MC>(c4[0], c4[1], c4[2]);
    hr = dev::half_slope<dev::LIM_MC>(c4[1], c4[2], c4[3]);
  } else if (lim == 2) {
    hl = dev::half_slope<dev::LIM_MM>(c4[0], c4[1], c4[2]);
    hr = dev::half_slope<dev::LIM_MM>(c4[1], c4[2], c4[3]);
  } else {
    hl = dev::half_slope<dev::LIM_VL>(c4[0], c4[1], c4[2]);
    hr = dev::half_slope<dev::LIM_VL>(c4[1], c4[2], c4[3]);
  }
  out[0] = c4[1] + hl;
  out[1] = c4[2] - hr;
}

void t_vjp_plm(int lim, const double* c4, double wLb, double wRb, double* cb) {
  adj::vjp_plm(lim, c4[0], c4[1], c4[2], c4[3], wLb, wRb, cb);
}

// characteristic-projected half slope of the cell wc (lim: 0 vl, 1 mc, 2 mm):
// the device forward (which = 0) or the adjoint header's restatement (which = 1)
void t_slopes_char(int which, int lim, const double* wm, const double* wc, const double* wp, double gam, double* d) {
  if (which == 1) {
    adj::slopes_char(lim, wm, wc, wp, gam, d);
  } else if (lim == 1) {
    dev::half_slopes_char<dev::LIM_MC>(wm, wc, wp, gam, d);
  } else if (lim == 2) {
    dev::half_slopes_char<dev::LIM_MM>(wm, wc, wp, gam, d);
  } else {
    dev::half_slopes_char<dev::LIM_VL>(wm, wc, wp, gam, d);
  }
}

void t_vjp_slopes_char(int lim, const double* wm, const double* wc, const double* wp, double gam, const double* db,
                       double* wmb, double* wcb, double* wpb) {
  for (int n = 0; n < 9; ++n) wmb[n] = wcb[n] = wpb[n] = 0.;
  adj::vjp_slopes_char(lim, wm, wc, wp, gam, db, wmb, wcb, wpb);
}

}  // extern "C"
