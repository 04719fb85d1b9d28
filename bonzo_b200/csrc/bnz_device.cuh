// bnz_device.cuh -- per-point device math of the VL2 step (FP64).
//
// EOS, fast magnetosonic speed, Riemann solvers (HLL, HLLT, HLLD; HLLC for
// the hydro system), slope limiters and PLM reconstruction of one interface.
// Every expression keeps the evaluation order of the reference's C kernels
// (src/mhd/eos_c.h, src/mhd/fluxes_c.c, src/coordinates/reconstr_c.{c,h}) so
// that a build with --fmad=false reproduces them bit for bit; the default
// build lets the compiler contract multiply-adds into DFMA.
//
// This header is included inside a namespace by bnz_kernels_impl.cuh, once per
// floating-point mode.
#pragma once

#include "bnz_fastmath.cuh"

#ifndef BNZ_NM
#define BNZ_NM 9
#endif

namespace dev {

constexpr int NM = 9;
enum { RHO = 0, MX = 1, MY = 2, MZ = 3, EN = 4, PSC = 5, BX = 6, BY = 7, BZ = 8 };
enum { VX = 1, VY = 2, VZ = 3, PR = 4 };
enum { RS_HLL = 0, RS_HLLC = 1, RS_HLLD = 2, RS_HLLT = 3 };
// HLL of the hydro build (MFIELD 0): the hydro sound speed in its wave
// estimate.  Internal code, not an ABI value.
enum { RS_HLL_HYDRO = 4 };
enum { LIM_VL = 0, LIM_MC = 1, LIM_MM = 2 };
// bits of the device error word
enum { ERR_RHO = 1, ERR_PRES = 2, ERR_NAN = 4, ERR_FAN = 8, ERR_TIMEOUT = 16 };

__device__ __forceinline__ double sqr(double x) { return x * x; }
__device__ __forceinline__ double sgnd(double a) { return (double)((0.0 < a) - (a < 0.0)); }

// eos_c.h:20-55 (MHD, no CGL / two-temperature terms)
__device__ __forceinline__ void cons2prim(double* w, const double* u, double gam) {
  double rhoi = 1. / u[RHO];
  w[RHO] = u[RHO];
  w[VX] = u[MX] * rhoi;
  w[VY] = u[MY] * rhoi;
  w[VZ] = u[MZ] * rhoi;
  double v2 = sqr(w[VX]) + sqr(w[VY]) + sqr(w[VZ]);
  double b2 = sqr(u[BX]) + sqr(u[BY]) + sqr(u[BZ]);
  w[PR] = (gam - 1.) * (u[EN] - 0.5 * (b2 + v2 * u[RHO]));
  w[PSC] = u[PSC];
  w[BX] = u[BX];
  w[BY] = u[BY];
  w[BZ] = u[BZ];
}

// eos_c.h:60-95
__device__ __forceinline__ void prim2cons(double* u, const double* w, double gam) {
  double gamm1i = 1. / (gam - 1.);
  u[RHO] = w[RHO];
  u[MX] = w[RHO] * w[VX];
  u[MY] = w[RHO] * w[VY];
  u[MZ] = w[RHO] * w[VZ];
  double v2 = sqr(w[VX]) + sqr(w[VY]) + sqr(w[VZ]);
  double b2 = sqr(w[BX]) + sqr(w[BY]) + sqr(w[BZ]);
  u[EN] = 0.5 * (w[RHO] * v2 + b2) + w[PR] * gamm1i;
  u[PSC] = w[PSC];
  u[BX] = w[BX];
  u[BY] = w[BY];
  u[BZ] = w[BZ];
}

// eos_c.h:416-461 with a = 1 (no pressure anisotropy)
__device__ __forceinline__ void primcons2flux(double* f, const double* w, const double* u) {
  double bx2 = sqr(w[BX]);
  double b2 = bx2 + sqr(w[BY]) + sqr(w[BZ]);
  double bxby = w[BX] * w[BY];
  double bxbz = w[BX] * w[BZ];
  double ptot = 0.5 * b2 + w[PR];
#pragma unroll
  for (int n = 0; n < BX; ++n) f[n] = u[n] * w[VX];
  f[MX] += ptot;
  f[EN] += ptot * w[VX];
  f[MX] -= bx2;
  f[MY] -= bxby;
  f[MZ] -= bxbz;
  f[EN] -= (w[VX] * bx2 + w[VY] * bxby + w[VZ] * bxbz);
  f[BX] = 0.;
  f[BY] = w[VX] * w[BY] - w[VY] * w[BX];
  f[BZ] = w[VX] * w[BZ] - w[VZ] * w[BX];
}

// eos_c.h:468-530 -- the normal field is read from w[BX] (the reference's
// bx argument is unused, so the CFL estimate uses the x fast speed on every axis).
__device__ __forceinline__ double fms(const double* w, double gam) {
  double bx2 = sqr(w[BX]);
  double b2 = bx2 + sqr(w[BY]) + sqr(w[BZ]);
  double gamp = gam * w[PR];
  double c1 = gamp + b2;
  double c2 = sqrt(fabs(c1 * c1 - 4. * gamp * bx2));
  return sqrt(0.5 / w[RHO] * (c1 + c2));
}

// 1/x: an IEEE division, or with NR in the fast build the Newton-refined
// reciprocal of bnz_fastmath.cuh (within 2 ulp, for normal finite x)
template <bool NR>
__device__ __forceinline__ double rcp_nr(double x) {
#if BNZ_FAST_MATH
  if constexpr (NR) return bnz_nr_rcp(x);
#endif
  return 1. / x;
}

#if BNZ_FAST_MATH
// fms of both face states with one division for the two 0.5 / rho
template <bool NR = false>
__device__ __forceinline__ void fms2(const double* wL, const double* wR, double gam, double& cfL, double& cfR) {
  const double h = NR ? 0.5 * rcp_nr<NR>(wL[RHO] * wR[RHO]) : 0.5 / (wL[RHO] * wR[RHO]);
  double q[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double* w = s ? wR : wL;
    double bx2 = sqr(w[BX]);
    double b2 = bx2 + sqr(w[BY]) + sqr(w[BZ]);
    double gamp = gam * w[PR];
    double c1 = gamp + b2;
    double c2 = sqrt(fabs(c1 * c1 - 4. * gamp * bx2));
    q[s] = (s ? wL[RHO] : wR[RHO]) * h * (c1 + c2);
  }
  cfL = sqrt(q[0]);
  cfR = sqrt(q[1]);
}
#endif

// fluxes_c.c:25-42
template <bool NR = false>
__device__ __forceinline__ void wave_speeds(const double* wL, const double* wR, double gam,
                                            double& sL, double& sR) {
#if BNZ_FAST_MATH
  double cfL, cfR;
  fms2<NR>(wL, wR, gam, cfL, cfR);
#else
  double cfL = fms(wL, gam);
  double cfR = fms(wR, gam);
#endif
  double cf_max = fmax(cfL, cfR);
  sL = fmin(wL[VX], wR[VX]) - cf_max;
  sR = fmax(wL[VX], wR[VX]) + cf_max;
}

// fluxes_c.c:175-223
__device__ __forceinline__ void flux_hll(double* flux, const double* wL, const double* wR, double gam) {
  double uL[NM], uR[NM], fL[NM], fR[NM];
  prim2cons(uL, wL, gam);
  prim2cons(uR, wR, gam);
  primcons2flux(fL, wL, uL);
  primcons2flux(fR, wR, uR);
  double sL, sR;
  wave_speeds(wL, wR, gam, sL, sR);
  double aL = fmin(sL, 0.);
  double aR = fmax(sR, 0.);
  double aLaR = aL * aR;
  double aRmaLi = 1. / (aR - aL);
#pragma unroll
  for (int n = 0; n < NM; ++n) flux[n] = (aR * fL[n] - aL * fR[n] + aLaR * (uR[n] - uL[n])) * aRmaLi;
  flux[BX] = 0.;
}

// ---------------------------------------------------------------------------
// Hydro build (MFIELD 0).  The magnetic entries of every state are zero, so
// prim2cons, cons2prim and primcons2flux above give the hydro build's values
// (their field terms add exact zeros); only the signal speeds differ.
// ---------------------------------------------------------------------------

// eos_c.h:468-530, hydro branch: the adiabatic sound speed.
__device__ __forceinline__ double fms_hydro(const double* w, double gam) {
  const double gamp = gam * w[PR];
  return sqrt(gamp / w[RHO]);
}

// fluxes_c.c:25-42 with the hydro sound speed
__device__ __forceinline__ void wave_speeds_hydro(const double* wL, const double* wR, double gam, double& sL,
                                                  double& sR) {
  const double cfL = fms_hydro(wL, gam), cfR = fms_hydro(wR, gam);
  const double cf_max = fmax(cfL, cfR);
  sL = fmin(wL[VX], wR[VX]) - cf_max;
  sR = fmax(wL[VX], wR[VX]) + cf_max;
}

// fluxes_c.c:138-168: PVRS pressure-based wave speeds (Toro), used by HLLC.
__device__ __forceinline__ void wave_speeds_pvrs(const double* wL, const double* wR, double gam, double& sL,
                                                 double& sR) {
  const double g1gh = 0.5 * (gam + 1.) / gam;
  const double aL = fms_hydro(wL, gam), aR = fms_hydro(wR, gam);
  const double ptL = wL[PR], ptR = wR[PR];
  const double pvrs =
      fmax(0., 0.5 * (ptL + ptR) - 0.125 * (wR[VX] - wL[VX]) * (wL[RHO] + wR[RHO]) * (aL + aR));
  const double qL = pvrs < ptL ? 1. : sqrt(1. + g1gh * (pvrs / ptL - 1.));
  const double qR = pvrs < ptR ? 1. : sqrt(1. + g1gh * (pvrs / ptR - 1.));
  sL = wL[VX] - aL * qL;
  sR = wR[VX] + aR * qR;
}

// fluxes_c.c:175-223 in the hydro build: six conserved entries, hydro speeds.
__device__ __forceinline__ void flux_hll_hydro(double* flux, const double* wL, const double* wR, double gam) {
  double uL[NM], uR[NM], fL[NM], fR[NM];
  prim2cons(uL, wL, gam);
  prim2cons(uR, wR, gam);
  primcons2flux(fL, wL, uL);
  primcons2flux(fR, wR, uR);
  double sL, sR;
  wave_speeds_hydro(wL, wR, gam, sL, sR);
  const double aL = fmin(sL, 0.), aR = fmax(sR, 0.);
  const double aLaR = aL * aR;
  const double aRmaLi = 1. / (aR - aL);
#pragma unroll
  for (int n = 0; n < BX; ++n) flux[n] = (aR * fL[n] - aL * fR[n] + aLaR * (uR[n] - uL[n])) * aRmaLi;
  flux[BX] = flux[BY] = flux[BZ] = 0.;
}

// fluxes_c.c:232-327 (Toro's HLLC; hydro builds only).  The contact speed sM
// and star pressure come from both sides; the flux is z * F_side + sLR * p*
// terms of the side the contact leaves the interface on, with the side's own
// wave speed clipped at 0 -- the reference forms z_L F_L + z_R F_R with the
// other side's weight exactly 0, so one side per lane gives the same values.
__device__ __forceinline__ void flux_hllc(double* flux, const double* wL, const double* wR, double gam) {
  double sL, sR;
  wave_speeds_pvrs(wL, wR, gam, sL, sR);
  const double gamm1i = 1. / (gam - 1.);
  // the conserved rho and mx of both states (prim2cons, eos_c.h:60-95)
  const double mxL = wL[RHO] * wL[VX], mxR = wR[RHO] * wR[VX];
  double vLsL = wL[VX] - sL, vRsR = wR[VX] - sR;
  const double xL = wL[RHO] * vLsL, xR = wR[RHO] * vRsR;
  const double xRxLi = 1. / (xR - xL);
  const double yL = wL[PR] + mxL * vLsL, yR = wR[PR] + mxR * vRsR;
  const double sM = xRxLi * (yR - yL);
  const double pts = xRxLi * (xR * yL - xL * yR);
  sL = fmin(sL, 0.);
  sR = fmax(sR, 0.);
  const bool left = sM > 0.;
  const double* w = left ? wL : wR;
  const double s = left ? sL : sR;
  const double v_s = w[VX] - s;
  const double ssMi = 1. / (s - sM);
  const double z = -sM * ssMi;
  const double sLR = s * ssMi;
  double u[NM];
  u[RHO] = w[RHO];
  u[MX] = w[RHO] * w[VX];
  u[MY] = w[RHO] * w[VY];
  u[MZ] = w[RHO] * w[VZ];
  const double v2 = sqr(w[VX]) + sqr(w[VY]) + sqr(w[VZ]);
  const double b2 = sqr(w[BX]) + sqr(w[BY]) + sqr(w[BZ]);
  u[EN] = 0.5 * (w[RHO] * v2 + b2) + w[PR] * gamm1i;
  u[PSC] = w[PSC];
  double f[BX];
#pragma unroll
  for (int n = 0; n < BX; ++n) f[n] = u[n] * v_s;
  f[MX] += w[PR];
  f[EN] += w[PR] * w[VX];
#pragma unroll
  for (int n = 0; n < BX; ++n) flux[n] = z * f[n];
  flux[MX] += sLR * pts;
  flux[EN] += sLR * pts * sM;
  flux[BX] = flux[BY] = flux[BZ] = 0.;
}

// fluxes_c.c:447-607 (Mignone 2012 isothermal-type three-wave solver).  The
// reference leaves the energy entries of its star states uninitialised; they
// are zero here.
__device__ __forceinline__ void flux_hllt(double* flux, const double* wL, const double* wR, double gam,
                                          unsigned& err) {
  double uL[NM], uR[NM], fL[NM], fR[NM];
  prim2cons(uL, wL, gam);
  prim2cons(uR, wR, gam);
  primcons2flux(fL, wL, uL);
  primcons2flux(fR, wR, uR);
  double sL, sR;
  wave_speeds(wL, wR, gam, sL, sR);
  double bx = wL[BX];
  double sRsLi = 1. / (sR - sL);
  double rhos = (sR * uR[RHO] - sL * uL[RHO] - (fR[RHO] - fL[RHO])) * sRsLi;
  double mxs = (sR * uR[MX] - sL * uL[MX] - (fR[MX] - fL[MX])) * sRsLi;
  double frhos = (sR * fL[RHO] - sL * fR[RHO] + sR * sL * (uR[RHO] - uL[RHO])) * sRsLi;
  double us = frhos / rhos;
  double pscs = (sR * uR[PSC] - sL * uL[PSC] - (fR[PSC] - fL[PSC])) * sRsLi;
  double uLs[NM], uRs[NM], uCs[NM];
#pragma unroll
  for (int n = 0; n < NM; ++n) { uLs[n] = 0.; uRs[n] = 0.; uCs[n] = 0.; }
  uLs[RHO] = rhos; uRs[RHO] = rhos;
  uLs[MX] = mxs;   uRs[MX] = mxs;
  uLs[PSC] = pscs; uRs[PSC] = pscs;
  uLs[MY] = rhos * wL[VY];
  uRs[MY] = rhos * wR[VY];
  uLs[MZ] = rhos * wL[VZ];
  uRs[MZ] = rhos * wR[VZ];
  double sLs = us, sRs = us;
  double rhosi = 1. / rhos;
  double sqrt_rhosi = sqrt(rhosi);
  sLs -= fabs(bx) * sqrt_rhosi;
  sRs += fabs(bx) * sqrt_rhosi;
  double xL = 1. / ((sL - sLs) * (sL - sRs));
  double xR = 1. / ((sR - sLs) * (sR - sRs));
  double yL = bx * xL * (us - wL[VX]);
  double yR = bx * xR * (us - wR[VX]);
  uLs[MY] -= yL * wL[BY];
  uRs[MY] -= yR * wR[BY];
  uLs[MZ] -= yL * wL[BZ];
  uRs[MZ] -= yR * wR[BZ];
  yL = (wL[RHO] * sqr(sL - wL[VX]) - sqr(bx)) * rhosi * xL;
  yR = (wR[RHO] * sqr(sR - wR[VX]) - sqr(bx)) * rhosi * xR;
  uLs[BY] = yL * wL[BY];
  uRs[BY] = yR * wR[BY];
  uLs[BZ] = yL * wL[BZ];
  uRs[BZ] = yR * wR[BZ];
  uCs[RHO] = rhos;
  uCs[MX] = mxs;
  uCs[PSC] = pscs;
  double sgnb = sgnd(bx);
  double x = 0.5 * sgnb / sqrt_rhosi;
  uCs[MY] = 0.5 * (uLs[MY] + uRs[MY]) + x * (uRs[BY] - uLs[BY]);
  uCs[MZ] = 0.5 * (uLs[MZ] + uRs[MZ]) + x * (uRs[BZ] - uLs[BZ]);
  uCs[BY] = 0.5 * (uLs[BY] + uRs[BY]) + x * rhosi * (uRs[MY] - uLs[MY]);
  uCs[BZ] = 0.5 * (uLs[BZ] + uRs[BZ]) + x * rhosi * (uRs[MZ] - uLs[MZ]);
  // sequential region tests of the reference; the last match wins
  int r = 0;
  if (sL > 0.) r = 1;
  if (sL <= 0. && 0. < sLs) r = 2;
  if (sLs <= 0. && 0. < sRs) r = 3;
  if (sRs <= 0. && 0. < sR) r = 4;
  if (sR <= 0.) r = 5;
  if (r == 0) err |= ERR_FAN;
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    double v;
    if (r == 1) v = fL[n];
    else if (r == 2) v = fL[n] + sL * (uLs[n] - uL[n]);
    else if (r == 3) v = fL[n] + sL * (uLs[n] - uL[n]) + sLs * (uCs[n] - uLs[n]);
    else if (r == 4) v = fR[n] + sR * (uRs[n] - uR[n]);
    else if (r == 5) v = fR[n];
    else v = 0.;
    flux[n] = v;
  }
  flux[BX] = 0.;
}

// fluxes_c.c:616-834 (Miyoshi & Kusano 2005 HLLD).
// Every value is computed by the reference's expression, but the state and
// flux vectors are built for ONE side only: regions 1-3 of the wave fan use
// the left states (fL, uL*, uL**), regions 4-6 the right ones with the same
// formulas.  The scalar star quantities (sM, p*, tangential star velocities
// and fields) are formed for both sides, the side is chosen per lane, and the
// 9-vectors are evaluated once -- about half the live registers of forming
// both sides, with no warp divergence.  NR (fast build only): the five
// reciprocals by bnz_nr_rcp instead of IEEE divisions.
template <bool NR = false>
__device__ __forceinline__ void flux_hlld(double* flux, const double* wL, const double* wR, double gam,
                                          unsigned& err) {
  const double bx = wL[BX];
  const double bx2 = sqr(bx);
  // pieces of prim2cons / primcons2flux that the HLL average needs
  const double b2L = bx2 + sqr(wL[BY]) + sqr(wL[BZ]);
  const double b2R = bx2 + sqr(wR[BY]) + sqr(wR[BZ]);
  const double ptL = wL[PR] + 0.5 * b2L;  // = primcons2flux's ptot (same operands)
  const double ptR = wR[PR] + 0.5 * b2R;
  const double mxL = wL[RHO] * wL[VX], mxR = wR[RHO] * wR[VX];  // u[MX] = f[RHO]
  const double fmxL = mxL * wL[VX] + ptL - bx2;                   // f[MX]
  const double fmxR = mxR * wR[VX] + ptR - bx2;
  double sL, sR;
  wave_speeds<NR>(wL, wR, gam, sL, sR);

  double deni = rcp_nr<NR>(sR * wR[RHO] - sL * wL[RHO] - (mxR - mxL));
  double sM = (sR * mxR - sL * mxL - (fmxR - fmxL)) * deni;

  double sLvxL = sL - wL[VX];
  double sRvxR = sR - wR[VX];
#if BNZ_FAST_MATH
  // one division for both reciprocals (sL < sM < sR)
  const double dLM = sL - sM, dRM = sR - sM;
  const double inv2 = rcp_nr<NR>(dLM * dRM);
  double sLsMi = dRM * inv2;
  double sRsMi = dLM * inv2;
#else
  double sLsMi = 1. / (sL - sM);
  double sRsMi = 1. / (sR - sM);
#endif
  double xL = sLvxL * sLsMi;
  double xR = sRvxR * sRsMi;
  double rLs = wL[RHO] * xL, rRs = wR[RHO] * xR;
  double pts = wL[RHO] * sLvxL * (sM - wL[VX]) + ptL;

  double rhosLvxL = wL[RHO] * sLvxL;
  double rhosRvxR = wR[RHO] * sRvxR;
#if BNZ_FAST_MATH
  const double DL = rhosLvxL * (sL - sM) - bx2, DR = rhosRvxR * (sR - sM) - bx2;
  const double iD = rcp_nr<NR>(DL * DR);
  double wvbL = DR * iD;
  double wvbR = DL * iD;
#else
  double wvbL = 1. / (rhosLvxL * (sL - sM) - bx2);
  double wvbR = 1. / (rhosRvxR * (sR - sM) - bx2);
#endif
  double wvL = bx * (sM - wL[VX]) * wvbL;
  double wvR = bx * (sM - wR[VX]) * wvbR;
  double vyLs = wL[VY] - wL[BY] * wvL;
  double vyRs = wR[VY] - wR[BY] * wvR;
  double vzLs = wL[VZ] - wL[BZ] * wvL;
  double vzRs = wR[VZ] - wR[BZ] * wvR;
  double wbL = (rhosLvxL * sLvxL - bx2) * wvbL;
  double wbR = (rhosRvxR * sRvxR - bx2) * wvbR;
  double byLs = wL[BY] * wbL, byRs = wR[BY] * wbR;
  double bzLs = wL[BZ] * wbL, bzRs = wR[BZ] * wbR;
  double vsbsL = sM * bx + vyLs * byLs + vzLs * bzLs;
  double vsbsR = sM * bx + vyRs * byRs + vzRs * bzRs;

#if BNZ_FAST_MATH
  const double isrL = rsqrt(rLs), isrR = rsqrt(rRs);
  double sqrt_rhoLs = rLs * isrL;
  double sqrt_rhoRs = rRs * isrR;
  double sLs = sM - fabs(bx) * isrL;
  double sRs = sM + fabs(bx) * isrR;
#else
  double sqrt_rhoLs = sqrt(rLs);
  double sqrt_rhoRs = sqrt(rRs);
  double sLs = sM - fabs(bx) / sqrt_rhoLs;
  double sRs = sM + fabs(bx) / sqrt_rhoRs;
#endif

  int r = 0;
  if (sL > 0.) r = 1;
  if (sL <= 0. && 0. < sLs) r = 2;
  if (sLs <= 0. && 0. < sM) r = 3;
  if (sM <= 0. && 0. < sRs) r = 4;
  if (sRs <= 0. && 0. < sR) r = 5;
  if (sR <= 0.) r = 6;
  if (r == 0) err |= ERR_FAN;

  // double-star tangential state (needs both sides)
  double rhoLRi = rcp_nr<NR>(sqrt_rhoLs + sqrt_rhoRs);
  double sgnb = sgnd(bx);
  double vyss = (sqrt_rhoLs * vyLs + sqrt_rhoRs * vyRs + (byRs - byLs) * sgnb) * rhoLRi;
  double vzss = (sqrt_rhoLs * vzLs + sqrt_rhoRs * vzRs + (bzRs - bzLs) * sgnb) * rhoLRi;
  double byss = (sqrt_rhoLs * byRs + sqrt_rhoRs * byLs + sqrt_rhoLs * sqrt_rhoRs * (vyRs - vyLs) * sgnb) * rhoLRi;
  double bzss = (sqrt_rhoLs * bzRs + sqrt_rhoRs * bzLs + sqrt_rhoLs * sqrt_rhoRs * (vzRs - vzLs) * sgnb) * rhoLRi;
  double vssbss = sM * bx + vyss * byss + vzss * bzss;

  // one side: L for regions 1-3, R for 4-6
  const bool left = r <= 3;
  double w[NM];
#pragma unroll
  for (int n = 0; n < NM; ++n) w[n] = left ? wL[n] : wR[n];
  const double s_o = left ? sL : sR;          // outer wave
  const double s_i = left ? sLs : sRs;        // Alfven wave
  const double x = left ? xL : xR;
  const double svx = left ? sLvxL : sRvxR;
  const double sMi = left ? sLsMi : sRsMi;
  const double pt = left ? ptL : ptR;
  const double rs = left ? rLs : rRs;
  const double vys = left ? vyLs : vyRs, vzs = left ? vzLs : vzRs;
  const double bys = left ? byLs : byRs, bzs = left ? bzLs : bzRs;
  const double vsbs = left ? vsbsL : vsbsR;
  const double srs = left ? sqrt_rhoLs : sqrt_rhoRs;

  double u[NM], f[NM];
  prim2cons(u, w, gam);
  primcons2flux(f, w, u);
  // single-star state (fluxes_c.c:690-760)
  double es = (svx * u[EN] - pt * w[VX] + pts * sM + bx * (w[VX] * bx + w[VY] * w[BY] + w[VZ] * w[BZ] - vsbs)) * sMi;
  const double us[NM] = {rs, rs * sM, rs * vys, rs * vzs, es, u[PSC] * x, 0., bys, bzs};
  // double-star state (fluxes_c.c:764-812)
  double t = srs * (vsbs - vssbss) * sgnb;
  double ess = left ? es - t : es + t;
  const double uss[NM] = {rs, rs * sM, rs * vyss, rs * vzss, ess, u[PSC] * x, 0., byss, bzss};
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    double v;
    if (r == 1 || r == 6) v = f[n];
    else if (r == 2 || r == 5) v = f[n] + s_o * (us[n] - u[n]);
    else if (r == 3 || r == 4) v = f[n] + s_o * (us[n] - u[n]) + s_i * (uss[n] - us[n]);
    else v = 0.;
    flux[n] = v;
  }
  flux[BX] = 0.;
}

// eos_c.h:100-216 prim2char (MHD): the differences vc (local sweep frame) in
// the characteristic basis of the state w; PSC and BX pass through.
__device__ __forceinline__ void prim2char(double* vc, const double* w, double gam) {
  const double vc_rho = vc[RHO], vc_vx = vc[VX], vc_vy = vc[VY], vc_vz = vc[VZ];
  const double vc_p = vc[PR], vc_by = vc[BY], vc_bz = vc[BZ];
  const double w_rho = w[RHO], w_p = w[PR], w_bx = w[BX], w_by = w[BY], w_bz = w[BZ];
  double rhoi = 1. / w_rho;
  double s = sgnd(w_bx);
  double a2rho = gam * w_p;
  double a = sqrt(a2rho * rhoi);
  double bx2 = sqr(w_bx);
  double bperp2 = sqr(w_by) + sqr(w_bz);
  double b2 = bx2 + bperp2;
  double x = a2rho + b2;
  double y = sqrt(fabs(x * x - 4. * a2rho * bx2));
  double cf2rho = 0.5 * (x + y);
  double cs2rho = 0.5 * (x - y);
  double cf = sqrt(rhoi * cf2rho);
  double cs = sqrt(rhoi * fabs(cs2rho));
  double z = 1. / (cf2rho - cs2rho);
  double alphaf, alphas;
  if (cf <= cs) {
    alphaf = 1.;
    alphas = 0.;
  } else if (a <= cs) {
    alphaf = 0.;
    alphas = 1.;
  } else if (cf <= a) {
    alphaf = 1.;
    alphas = 0.;
  } else {
    alphaf = sqrt(z * fabs(a2rho - cs2rho));
    alphas = sqrt(z * fabs(cf2rho - a2rho));
  }
  double nf = 0.5 / (a2rho * rhoi);
  double qf_ = nf * cf * alphaf * s;
  double qs_ = nf * cs * alphas * s;
  double alphaf_ = nf * alphaf;
  double alphas_ = nf * alphas;
  double rhoisr = sqrt(rhoi);
  double arhoisr = a * rhoisr;
  double Af_ = alphaf_ * arhoisr;
  double As_ = alphas_ * arhoisr;
  x = s * rhoisr;
  double betay = 0., betaz = 0.;
  if (bperp2 != 0.) {
    double bperpi = 1. / sqrt(bperp2);
    betay = bperpi * w_by;
    betaz = bperpi * w_bz;
  }
  vc[RHO] = (alphaf_ * (rhoi * vc_p - cf * vc_vx) + qs_ * (betay * vc_vy + betaz * vc_vz) +
             As_ * (betay * vc_by + betaz * vc_bz));
  vc[VX] = 0.5 * ((-betaz * vc_vy + betay * vc_vz) + x * (-betaz * vc_by + betay * vc_bz));
  vc[VY] = (alphas_ * (rhoi * vc_p - cs * vc_vx) - qf_ * (betay * vc_vy + betaz * vc_vz) -
            Af_ * (betay * vc_by + betaz * vc_bz));
  vc[VZ] = vc_rho - 2. * nf * vc_p;
  vc[PR] = (alphas_ * (rhoi * vc_p + cs * vc_vx) + qf_ * (betay * vc_vy + betaz * vc_vz) -
            Af_ * (betay * vc_by + betaz * vc_bz));
  vc[BY] = 0.5 * ((betaz * vc_vy - betay * vc_vz) + x * (-betaz * vc_by + betay * vc_bz));
  vc[BZ] = (alphaf_ * (rhoi * vc_p + cf * vc_vx) - qs_ * (betay * vc_vy + betaz * vc_vz) +
            As_ * (betay * vc_by + betaz * vc_bz));
}

// eos_c.h:245-333 char2prim (MHD): back to primitive differences.
__device__ __forceinline__ void char2prim(double* vc, const double* w, double gam) {
  const double vc_rho = vc[RHO], vc_vx = vc[VX], vc_vy = vc[VY], vc_vz = vc[VZ];
  const double vc_p = vc[PR], vc_by = vc[BY], vc_bz = vc[BZ];
  const double w_rho = w[RHO], w_p = w[PR], w_bx = w[BX], w_by = w[BY], w_bz = w[BZ];
  double rhoi = 1. / w_rho;
  double s = sgnd(w_bx);
  double a2rho = gam * w_p;
  double a = sqrt(a2rho * rhoi);
  double bx2 = sqr(w_bx);
  double bperp2 = sqr(w_by) + sqr(w_bz);
  double b2 = bx2 + bperp2;
  double x = a2rho + b2;
  double y = sqrt(fabs(x * x - 4. * a2rho * bx2));
  double cf2rho = 0.5 * (x + y);
  double cs2rho = 0.5 * (x - y);
  double cf = sqrt(rhoi * cf2rho);
  double cs = sqrt(rhoi * fabs(cs2rho));
  double z = 1. / (cf2rho - cs2rho);
  double alphaf, alphas;
  if (cf <= cs) {
    alphaf = 1.;
    alphas = 0.;
  } else if (a <= cs) {
    alphaf = 0.;
    alphas = 1.;
  } else if (cf <= a) {
    alphaf = 1.;
    alphas = 0.;
  } else {
    alphaf = sqrt(z * fabs(a2rho - cs2rho));
    alphas = sqrt(z * fabs(cf2rho - a2rho));
  }
  double qf = cf * alphaf * s;
  double qs = cs * alphas * s;
  double rhosr = sqrt(w_rho);
  double arhosr = a * rhosr;
  double Af = alphaf * arhosr;
  double As = alphas * arhosr;
  double betay = 0., betaz = 0.;
  if (bperp2 != 0.) {
    double bperpi = 1. / sqrt(bperp2);
    betay = bperpi * w_by;
    betaz = bperpi * w_bz;
  }
  vc[RHO] = w_rho * (alphaf * (vc_rho + vc_bz) + alphas * (vc_vy + vc_p)) + vc_vz;
  vc[VX] = cf * alphaf * (vc_bz - vc_rho) + cs * alphas * (vc_p - vc_vy);
  vc[VY] = betay * (qs * (vc_rho - vc_bz) - qf * (vc_vy - vc_p)) - betaz * (vc_vx - vc_by);
  vc[VZ] = betaz * (qs * (vc_rho - vc_bz) - qf * (vc_vy - vc_p)) + betay * (vc_vx - vc_by);
  vc[PR] = a2rho * (alphaf * (vc_rho + vc_bz) + alphas * (vc_vy + vc_p));
  vc[BY] = betay * (As * (vc_rho + vc_bz) - Af * (vc_vy + vc_p)) - betaz * s * rhosr * (vc_vx + vc_by);
  vc[BZ] = betaz * (As * (vc_rho + vc_bz) - Af * (vc_vy + vc_p)) + betay * s * rhosr * (vc_vx + vc_by);
}

// NR: the fast build's HLLD takes its reciprocals by bnz_nr_rcp
template <int RS, bool NR = false>
__device__ __forceinline__ void riemann(double* flux, const double* wL, const double* wR, double gam,
                                        unsigned& err) {
  if constexpr (RS == RS_HLLD) flux_hlld<NR>(flux, wL, wR, gam, err);
  else if constexpr (RS == RS_HLLT) flux_hllt(flux, wL, wR, gam, err);
  else if constexpr (RS == RS_HLLC) flux_hllc(flux, wL, wR, gam);
  else if constexpr (RS == RS_HLL_HYDRO) flux_hll_hydro(flux, wL, wR, gam);
  else flux_hll(flux, wL, wR, gam);
}

// reconstr_c.h:28-44
__device__ __forceinline__ double mm_lim(double a, double b) {
  return (a * b <= 0.) ? 0. : ((a > 0.) ? ((a < b) ? a : b) : ((a > b) ? a : b));
}
__device__ __forceinline__ double mc_lim(double a, double b) { return mm_lim(2. * mm_lim(a, b), 0.5 * (a + b)); }
__device__ __forceinline__ double vl_lim(double a, double b) {
  double ab = a * b;
  return (ab > 0.) ? (2. * ab / (a + b)) : 0.;
}
template <int LIM>
__device__ __forceinline__ double limit(double a, double b) {
  if constexpr (LIM == LIM_MC) return mc_lim(a, b);
  else if constexpr (LIM == LIM_MM) return mm_lim(a, b);
  else return vl_lim(a, b);
}

// reconstr_c.c:54-91 for one cell: half slope d = 0.5 lim(dm, dp); the face
// states are wc - d (left face of the cell) and wc + d (right face).
template <int LIM>
__device__ __forceinline__ double half_slope(double wm, double wc, double wp) {
  return 0.5 * limit<LIM>(wc - wm, wp - wc);
}

// reconstr_c.c:54-91 with charact_proj: the one-sided differences of all nine
// local variables are projected on the characteristic basis of the cell
// (prim2char), limited, scaled by 1/2 and projected back (char2prim).
template <int LIM>
__device__ __forceinline__ void half_slopes_char(const double* wm, const double* wc, const double* wp, double gam,
                                                 double* d) {
  double dm[NM], dp[NM];
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    dm[n] = wc[n] - wm[n];
    dp[n] = wp[n] - wc[n];
  }
  prim2char(dm, wc, gam);
  prim2char(dp, wc, gam);
#pragma unroll
  for (int n = 0; n < NM; ++n) d[n] = 0.5 * limit<LIM>(dm[n], dp[n]);
  char2prim(d, wc, gam);
}

}  // namespace dev
