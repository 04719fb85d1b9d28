// bnz_adjoint_math.h -- pointwise vector-Jacobian products (reverse mode) of
// the per-point math of the VL2 step: EOS conversions, the ideal-MHD flux,
// the fast magnetosonic speed, the HLL, HLLT and HLLD Riemann solvers and
// the PLM slope limiters.  Hand-derived from the forward expressions in
// bnz_device.cuh (which restate src/mhd/eos_c.h, src/mhd/fluxes_c.c and
// src/coordinates/reconstr_c.h); the reference has no adjoint.
//
// Every function takes the forward inputs, recomputes what it needs and adds
// (+=) the input cotangents; the branch taken at a kink (limiter cases, the
// Riemann fan region, min/max of wave speeds, |x|) is the one the forward
// takes for the same inputs.  Variables are in the sweep's local frame with
// the layout of dev::NM (RHO, VX, VY, VZ, PR, PSC, BX, BY, BZ); the normal
// field is w[BX] on both sides and its cotangent is returned separately.
//
// The header compiles as CUDA device code (included inside the kernels'
// namespace) and as plain C++ for host-side tests.
#pragma once

#ifdef __CUDACC__
#define BNZ_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define BNZ_HD inline
#endif

namespace adj {

enum { RHO = 0, VX = 1, VY = 2, VZ = 3, PR = 4, PSC = 5, BX = 6, BY = 7, BZ = 8 };
enum { MX = 1, MY = 2, MZ = 3, EN = 4 };
constexpr int NM = 9;

BNZ_HD double sq(double x) { return x * x; }
BNZ_HD double sgn(double a) { return (double)((0.0 < a) - (a < 0.0)); }

// a / b: in the fast build's device code a times the Newton-refined
// reciprocal the forward HLLD uses (bnz_fastmath.cuh), elsewhere the IEEE
// quotient
BNZ_HD double quo(double a, double b) {
#if BNZ_FAST_MATH && defined(__CUDA_ARCH__)
  return a * bnz_nr_rcp(b);
#else
  return a / b;
#endif
}

// w = cons2prim(u): given wbar, add ubar.  Expressed through w (the forward's
// output), which holds rho, v and B.
BNZ_HD void vjp_cons2prim(const double* w, const double* wb, double gam, double* ub) {
  const double g1 = gam - 1.;
  const double rhoi = 1. / w[RHO];
  const double pb = wb[PR];
  const double v2 = sq(w[VX]) + sq(w[VY]) + sq(w[VZ]);
  ub[EN] += g1 * pb;
  ub[RHO] += wb[RHO] - (wb[VX] * w[VX] + wb[VY] * w[VY] + wb[VZ] * w[VZ]) * rhoi + 0.5 * g1 * v2 * pb;
  ub[MX] += wb[VX] * rhoi - g1 * w[VX] * pb;
  ub[MY] += wb[VY] * rhoi - g1 * w[VY] * pb;
  ub[MZ] += wb[VZ] * rhoi - g1 * w[VZ] * pb;
  ub[PSC] += wb[PSC];
  ub[BX] += wb[BX] - g1 * w[BX] * pb;
  ub[BY] += wb[BY] - g1 * w[BY] * pb;
  ub[BZ] += wb[BZ] - g1 * w[BZ] * pb;
}

// u = prim2cons(w): given ubar, add wbar.
BNZ_HD void vjp_prim2cons(const double* w, const double* ub, double gam, double* wb) {
  const double gamm1i = 1. / (gam - 1.);
  const double eb = ub[EN];
  const double v2 = sq(w[VX]) + sq(w[VY]) + sq(w[VZ]);
  wb[RHO] += ub[RHO] + ub[MX] * w[VX] + ub[MY] * w[VY] + ub[MZ] * w[VZ] + 0.5 * v2 * eb;
  wb[VX] += ub[MX] * w[RHO] + eb * w[RHO] * w[VX];
  wb[VY] += ub[MY] * w[RHO] + eb * w[RHO] * w[VY];
  wb[VZ] += ub[MZ] * w[RHO] + eb * w[RHO] * w[VZ];
  wb[PR] += eb * gamm1i;
  wb[PSC] += ub[PSC];
  wb[BX] += ub[BX] + eb * w[BX];
  wb[BY] += ub[BY] + eb * w[BY];
  wb[BZ] += ub[BZ] + eb * w[BZ];
}

// f = flux(w) of ideal MHD along x (primcons2flux of prim2cons(w); f[BX] = 0):
// given fbar (entry BX ignored), add wbar; the w[BX] part goes to wb[BX].
BNZ_HD void vjp_flux(const double* w, const double* fb, double gam, double* wb) {
  const double r = w[RHO], vx = w[VX], vy = w[VY], vz = w[VZ], p = w[PR];
  const double bx = w[BX], by = w[BY], bz = w[BZ];
  const double b2 = sq(bx) + sq(by) + sq(bz);
  const double v2 = sq(vx) + sq(vy) + sq(vz);
  const double pt = p + 0.5 * b2;
  const double gamm1i = 1. / (gam - 1.);
  const double en = 0.5 * (r * v2 + b2) + p * gamm1i;
  const double dot = vx * bx + vy * by + vz * bz;
  double rb = 0., vxb = 0., vyb = 0., vzb = 0., pb = 0., bxb = 0., byb = 0., bzb = 0.;
  double ptb = 0., enb = 0.;
  // f[RHO] = r vx
  rb += fb[RHO] * vx;
  vxb += fb[RHO] * r;
  // f[MX] = r vx vx + pt - bx^2
  rb += fb[MX] * vx * vx;
  vxb += 2. * fb[MX] * r * vx;
  ptb += fb[MX];
  bxb -= 2. * fb[MX] * bx;
  // f[MY] = r vx vy - bx by
  rb += fb[MY] * vx * vy;
  vxb += fb[MY] * r * vy;
  vyb += fb[MY] * r * vx;
  bxb -= fb[MY] * by;
  byb -= fb[MY] * bx;
  // f[MZ] = r vx vz - bx bz
  rb += fb[MZ] * vx * vz;
  vxb += fb[MZ] * r * vz;
  vzb += fb[MZ] * r * vx;
  bxb -= fb[MZ] * bz;
  bzb -= fb[MZ] * bx;
  // f[EN] = (en + pt) vx - bx dot
  enb += fb[EN] * vx;
  ptb += fb[EN] * vx;
  vxb += fb[EN] * (en + pt);
  bxb -= fb[EN] * dot;
  {
    const double dotb = -fb[EN] * bx;
    vxb += dotb * bx;
    bxb += dotb * vx;
    vyb += dotb * by;
    byb += dotb * vy;
    vzb += dotb * bz;
    bzb += dotb * vz;
  }
  // f[PSC] = psc vx
  wb[PSC] += fb[PSC] * vx;
  vxb += fb[PSC] * w[PSC];
  // f[BY] = vx by - vy bx ; f[BZ] = vx bz - vz bx
  vxb += fb[BY] * by + fb[BZ] * bz;
  byb += fb[BY] * vx;
  vyb -= fb[BY] * bx;
  bxb -= fb[BY] * vy + fb[BZ] * vz;
  bzb += fb[BZ] * vx;
  vzb -= fb[BZ] * bx;
  // en = 0.5 (r v2 + b2) + p / (gam - 1)
  rb += enb * 0.5 * v2;
  vxb += enb * r * vx;
  vyb += enb * r * vy;
  vzb += enb * r * vz;
  bxb += enb * bx;
  byb += enb * by;
  bzb += enb * bz;
  pb += enb * gamm1i;
  // pt = p + 0.5 b2
  pb += ptb;
  bxb += ptb * bx;
  byb += ptb * by;
  bzb += ptb * bz;
  wb[RHO] += rb;
  wb[VX] += vxb;
  wb[VY] += vyb;
  wb[VZ] += vzb;
  wb[PR] += pb;
  wb[BX] += bxb;
  wb[BY] += byb;
  wb[BZ] += bzb;
}

// conserved vector u = prim2cons(w): value (for the Riemann VJPs)
BNZ_HD void cons_of(const double* w, double gam, double* u) {
  u[RHO] = w[RHO];
  u[MX] = w[RHO] * w[VX];
  u[MY] = w[RHO] * w[VY];
  u[MZ] = w[RHO] * w[VZ];
  u[EN] = 0.5 * (w[RHO] * (sq(w[VX]) + sq(w[VY]) + sq(w[VZ])) + sq(w[BX]) + sq(w[BY]) + sq(w[BZ])) +
          w[PR] / (gam - 1.);
  u[PSC] = w[PSC];
  u[BX] = w[BX];
  u[BY] = w[BY];
  u[BZ] = w[BZ];
}

BNZ_HD void flux_of(const double* w, double gam, double* f) {
  const double b2 = sq(w[BX]) + sq(w[BY]) + sq(w[BZ]);
  const double pt = w[PR] + 0.5 * b2;
  const double en = 0.5 * (w[RHO] * (sq(w[VX]) + sq(w[VY]) + sq(w[VZ])) + b2) + w[PR] / (gam - 1.);
  const double dot = w[VX] * w[BX] + w[VY] * w[BY] + w[VZ] * w[BZ];
  f[RHO] = w[RHO] * w[VX];
  f[MX] = w[RHO] * w[VX] * w[VX] + pt - sq(w[BX]);
  f[MY] = w[RHO] * w[VX] * w[VY] - w[BX] * w[BY];
  f[MZ] = w[RHO] * w[VX] * w[VZ] - w[BX] * w[BZ];
  f[EN] = (en + pt) * w[VX] - w[BX] * dot;
  f[PSC] = w[PSC] * w[VX];
  f[BX] = 0.;
  f[BY] = w[VX] * w[BY] - w[VY] * w[BX];
  f[BZ] = w[VX] * w[BZ] - w[VZ] * w[BX];
}

// cf = fms(w) (eos_c.h:468-530; the normal field is w[BX]): value and VJP.
BNZ_HD double fms_val(const double* w, double gam) {
  const double bx2 = sq(w[BX]);
  const double b2 = bx2 + sq(w[BY]) + sq(w[BZ]);
  const double gamp = gam * w[PR];
  const double c1 = gamp + b2;
  const double c2 = sqrt(fabs(c1 * c1 - 4. * gamp * bx2));
  return sqrt(quo(0.5, w[RHO]) * (c1 + c2));
}

// VJP of cf = fms(w) given its value cf (> 0)
BNZ_HD void vjp_fms(const double* w, double cf, double cfb, double gam, double* wb) {
  if (!(cf > 0.)) return;
  const double bx2 = sq(w[BX]);
  const double b2 = bx2 + sq(w[BY]) + sq(w[BZ]);
  const double gamp = gam * w[PR];
  const double c1 = gamp + b2;
  const double disc = c1 * c1 - 4. * gamp * bx2;
  const double c2 = sqrt(fabs(disc));
  const double rhoi = quo(1., w[RHO]);
  const double qb = quo(cfb * 0.5, cf);  // q = 0.5 / rho (c1 + c2)
  wb[RHO] += -qb * 0.5 * rhoi * rhoi * (c1 + c2);
  double c1b = qb * 0.5 * rhoi;
  const double c2b = c1b;
  double gampb = 0., bx2b = 0., b2b = 0.;
  if (c2 > 0.) {
    const double discb = quo(c2b * 0.5, c2) * sgn(disc);
    c1b += 2. * c1 * discb;
    gampb -= 4. * bx2 * discb;
    bx2b -= 4. * gamp * discb;
  }
  gampb += c1b;
  b2b += c1b;
  wb[PR] += gam * gampb;
  bx2b += b2b;
  wb[BY] += 2. * w[BY] * b2b;
  wb[BZ] += 2. * w[BZ] * b2b;
  wb[BX] += 2. * w[BX] * bx2b;
}

// sL = min(vxL, vxR) - max(cfL, cfR), sR = max(vxL, vxR) + max(cfL, cfR)
// (fluxes_c.c:25-42): VJP given sLb, sRb.
BNZ_HD void vjp_wave_speeds(const double* wL, const double* wR, double cfL, double cfR, double gam, double sLb,
                            double sRb, double* wLb, double* wRb) {
  const double cfmb = -sLb + sRb;
  // fmax / fmin pick the first argument on ties
  if (cfL >= cfR) vjp_fms(wL, cfL, cfmb, gam, wLb);
  else vjp_fms(wR, cfR, cfmb, gam, wRb);
  if (wL[VX] <= wR[VX]) wLb[VX] += sLb;
  else wRb[VX] += sLb;
  if (wL[VX] >= wR[VX]) wLb[VX] += sRb;
  else wRb[VX] += sRb;
}

// HLL flux (fluxes_c.c:175-223): given fb, add wLb, wRb (normal field into
// the BX entries of both; the caller sums them).
BNZ_HD void vjp_hll(const double* wL, const double* wR, double gam, const double* fb, double* wLb, double* wRb) {
  double uL[NM], uR[NM], fL[NM], fR[NM];
  cons_of(wL, gam, uL);
  cons_of(wR, gam, uR);
  flux_of(wL, gam, fL);
  flux_of(wR, gam, fR);
  const double cfL = fms_val(wL, gam), cfR = fms_val(wR, gam);
  const double cfm = cfL > cfR ? cfL : cfR;
  const double sL = (wL[VX] < wR[VX] ? wL[VX] : wR[VX]) - cfm;
  const double sR = (wL[VX] > wR[VX] ? wL[VX] : wR[VX]) + cfm;
  const double aL = sL < 0. ? sL : 0.;
  const double aR = sR > 0. ? sR : 0.;
  const double inv = 1. / (aR - aL);
  double fLb[NM], fRb[NM], uLb[NM], uRb[NM];
  double aLb = 0., aRb = 0., invb = 0.;
  for (int n = 0; n < NM; ++n) {
    const double fbn = n == BX ? 0. : fb[n];
    const double g = aR * fL[n] - aL * fR[n] + aL * aR * (uR[n] - uL[n]);
    const double gb = fbn * inv;
    invb += fbn * g;
    fLb[n] = gb * aR;
    fRb[n] = -gb * aL;
    uRb[n] = gb * aL * aR;
    uLb[n] = -gb * aL * aR;
    aRb += gb * fL[n] + gb * aL * (uR[n] - uL[n]);
    aLb += -gb * fR[n] + gb * aR * (uR[n] - uL[n]);
  }
  const double db = -invb * inv * inv;
  aRb += db;
  aLb -= db;
  const double sLb = sL < 0. ? aLb : 0.;
  const double sRb = sR > 0. ? aRb : 0.;
  vjp_flux(wL, fLb, gam, wLb);
  vjp_flux(wR, fRb, gam, wRb);
  vjp_prim2cons(wL, uLb, gam, wLb);
  vjp_prim2cons(wR, uRb, gam, wRb);
  vjp_wave_speeds(wL, wR, cfL, cfR, gam, sLb, sRb, wLb, wRb);
}

// HLLT flux (fluxes_c.c:447-607, as restated in bnz_device.cuh flux_hllt):
// given fb, add wLb, wRb (the normal field's cotangent goes to the BX entries
// of both sides; the caller sums them).  The star states' energy entries are
// zero, as in the forward.  The fan region is the one the forward selects;
// where it finds none (ERR_FAN) its flux is zero and so is the VJP.
BNZ_HD void vjp_hllt(const double* wL, const double* wR, double gam, const double* fb, double* wLb, double* wRb) {
  // ---- forward (values kept for the reverse sweep) ----
  double uL[NM], uR[NM], fL[NM], fR[NM];
  cons_of(wL, gam, uL);
  cons_of(wR, gam, uR);
  flux_of(wL, gam, fL);
  flux_of(wR, gam, fR);
  const double cfL = fms_val(wL, gam), cfR = fms_val(wR, gam);
  const double cfm = cfL > cfR ? cfL : cfR;
  const double sL = (wL[VX] < wR[VX] ? wL[VX] : wR[VX]) - cfm;
  const double sR = (wL[VX] > wR[VX] ? wL[VX] : wR[VX]) + cfm;
  const double bx = wL[BX], abx = fabs(bx);
  const double Di = 1. / (sR - sL);
  // HLL averages of rho, mx, the mass flux and the passive scalar
  const double nr = sR * uR[RHO] - sL * uL[RHO] - (fR[RHO] - fL[RHO]);
  const double nm = sR * uR[MX] - sL * uL[MX] - (fR[MX] - fL[MX]);
  const double nf = sR * fL[RHO] - sL * fR[RHO] + sR * sL * (uR[RHO] - uL[RHO]);
  const double np = sR * uR[PSC] - sL * uL[PSC] - (fR[PSC] - fL[PSC]);
  const double rhos = nr * Di, mxs = nm * Di, frhos = nf * Di, pscs = np * Di;
  const double us = frhos / rhos;
  const double rhosi = 1. / rhos;
  const double sqri = sqrt(rhosi);
  const double sLs = us - abx * sqri, sRs = us + abx * sqri;
  const double xL = 1. / ((sL - sLs) * (sL - sRs)), xR = 1. / ((sR - sLs) * (sR - sRs));
  const double y1L = bx * xL * (us - wL[VX]), y1R = bx * xR * (us - wR[VX]);
  const double AL = wL[RHO] * sq(sL - wL[VX]) - sq(bx), AR = wR[RHO] * sq(sR - wR[VX]) - sq(bx);
  const double y2L = AL * rhosi * xL, y2R = AR * rhosi * xR;
  double uLs[NM], uRs[NM], uCs[NM];
  for (int n = 0; n < NM; ++n) uLs[n] = uRs[n] = uCs[n] = 0.;
  uLs[RHO] = uRs[RHO] = uCs[RHO] = rhos;
  uLs[MX] = uRs[MX] = uCs[MX] = mxs;
  uLs[PSC] = uRs[PSC] = uCs[PSC] = pscs;
  uLs[MY] = rhos * wL[VY] - y1L * wL[BY];
  uRs[MY] = rhos * wR[VY] - y1R * wR[BY];
  uLs[MZ] = rhos * wL[VZ] - y1L * wL[BZ];
  uRs[MZ] = rhos * wR[VZ] - y1R * wR[BZ];
  uLs[BY] = y2L * wL[BY];
  uRs[BY] = y2R * wR[BY];
  uLs[BZ] = y2L * wL[BZ];
  uRs[BZ] = y2R * wR[BZ];
  const double x = 0.5 * sgn(bx) / sqri, xr = x * rhosi;
  uCs[MY] = 0.5 * (uLs[MY] + uRs[MY]) + x * (uRs[BY] - uLs[BY]);
  uCs[MZ] = 0.5 * (uLs[MZ] + uRs[MZ]) + x * (uRs[BZ] - uLs[BZ]);
  uCs[BY] = 0.5 * (uLs[BY] + uRs[BY]) + xr * (uRs[MY] - uLs[MY]);
  uCs[BZ] = 0.5 * (uLs[BZ] + uRs[BZ]) + xr * (uRs[MZ] - uLs[MZ]);
  int r = 0;
  if (sL > 0.) r = 1;
  if (sL <= 0. && 0. < sLs) r = 2;
  if (sLs <= 0. && 0. < sRs) r = 3;
  if (sRs <= 0. && 0. < sR) r = 4;
  if (sR <= 0.) r = 5;
  if (r == 0) return;
  // ---- reverse ----
  double fLb[NM], fRb[NM], uLb[NM], uRb[NM], uLsb[NM], uRsb[NM], uCsb[NM];
  for (int n = 0; n < NM; ++n) fLb[n] = fRb[n] = uLb[n] = uRb[n] = uLsb[n] = uRsb[n] = uCsb[n] = 0.;
  double sLb = 0., sRb = 0., sLsb = 0., sRsb = 0.;
  for (int n = 0; n < NM; ++n) {
    const double g = n == BX ? 0. : fb[n];
    if (r == 1) {
      fLb[n] += g;
    } else if (r == 2 || r == 3) {  // fL + sL (uL* - uL) [+ sL* (uC* - uL*)]
      fLb[n] += g;
      sLb += g * (uLs[n] - uL[n]);
      uLsb[n] += sL * g;
      uLb[n] -= sL * g;
      if (r == 3) {
        sLsb += g * (uCs[n] - uLs[n]);
        uCsb[n] += sLs * g;
        uLsb[n] -= sLs * g;
      }
    } else if (r == 4) {  // fR + sR (uR* - uR)
      fRb[n] += g;
      sRb += g * (uRs[n] - uR[n]);
      uRsb[n] += sR * g;
      uRb[n] -= sR * g;
    } else {
      fRb[n] += g;
    }
  }
  // central state
  double rhosb = uCsb[RHO], mxsb = uCsb[MX], pscsb = uCsb[PSC], xb = 0., xrb = 0.;
  {
    const double c = uCsb[MY];
    uLsb[MY] += 0.5 * c;
    uRsb[MY] += 0.5 * c;
    xb += c * (uRs[BY] - uLs[BY]);
    uRsb[BY] += c * x;
    uLsb[BY] -= c * x;
  }
  {
    const double c = uCsb[MZ];
    uLsb[MZ] += 0.5 * c;
    uRsb[MZ] += 0.5 * c;
    xb += c * (uRs[BZ] - uLs[BZ]);
    uRsb[BZ] += c * x;
    uLsb[BZ] -= c * x;
  }
  {
    const double c = uCsb[BY];
    uLsb[BY] += 0.5 * c;
    uRsb[BY] += 0.5 * c;
    xrb += c * (uRs[MY] - uLs[MY]);
    uRsb[MY] += c * xr;
    uLsb[MY] -= c * xr;
  }
  {
    const double c = uCsb[BZ];
    uLsb[BZ] += 0.5 * c;
    uRsb[BZ] += 0.5 * c;
    xrb += c * (uRs[MZ] - uLs[MZ]);
    uRsb[MZ] += c * xr;
    uLsb[MZ] -= c * xr;
  }
  xb += xrb * rhosi;
  double rhosib = xrb * x;
  double sqrib = -xb * x / sqri;  // x = 0.5 sgn(bx) / sqri
  // outer star states
  rhosb += uLsb[RHO] + uRsb[RHO];
  mxsb += uLsb[MX] + uRsb[MX];
  pscsb += uLsb[PSC] + uRsb[PSC];
  rhosb += uLsb[MY] * wL[VY] + uLsb[MZ] * wL[VZ] + uRsb[MY] * wR[VY] + uRsb[MZ] * wR[VZ];
  wLb[VY] += uLsb[MY] * rhos;
  wLb[VZ] += uLsb[MZ] * rhos;
  wRb[VY] += uRsb[MY] * rhos;
  wRb[VZ] += uRsb[MZ] * rhos;
  const double y1Lb = -(uLsb[MY] * wL[BY] + uLsb[MZ] * wL[BZ]);
  const double y1Rb = -(uRsb[MY] * wR[BY] + uRsb[MZ] * wR[BZ]);
  wLb[BY] += uLsb[BY] * y2L - uLsb[MY] * y1L;
  wLb[BZ] += uLsb[BZ] * y2L - uLsb[MZ] * y1L;
  wRb[BY] += uRsb[BY] * y2R - uRsb[MY] * y1R;
  wRb[BZ] += uRsb[BZ] * y2R - uRsb[MZ] * y1R;
  const double y2Lb = uLsb[BY] * wL[BY] + uLsb[BZ] * wL[BZ];
  const double y2Rb = uRsb[BY] * wR[BY] + uRsb[BZ] * wR[BZ];
  // y2 = (rho (s - vx)^2 - bx^2) / rho* x
  double bxb = 0., xLb = 0., xRb = 0., usb = 0.;
  {
    const double Ab = y2Lb * rhosi * xL;
    rhosib += y2Lb * AL * xL;
    xLb += y2Lb * AL * rhosi;
    wLb[RHO] += Ab * sq(sL - wL[VX]);
    const double t = Ab * wL[RHO] * 2. * (sL - wL[VX]);
    sLb += t;
    wLb[VX] -= t;
    bxb -= Ab * 2. * bx;
  }
  {
    const double Ab = y2Rb * rhosi * xR;
    rhosib += y2Rb * AR * xR;
    xRb += y2Rb * AR * rhosi;
    wRb[RHO] += Ab * sq(sR - wR[VX]);
    const double t = Ab * wR[RHO] * 2. * (sR - wR[VX]);
    sRb += t;
    wRb[VX] -= t;
    bxb -= Ab * 2. * bx;
  }
  // y1 = bx x (u* - vx)
  bxb += y1Lb * xL * (us - wL[VX]) + y1Rb * xR * (us - wR[VX]);
  xLb += y1Lb * bx * (us - wL[VX]);
  xRb += y1Rb * bx * (us - wR[VX]);
  usb += y1Lb * bx * xL + y1Rb * bx * xR;
  wLb[VX] -= y1Lb * bx * xL;
  wRb[VX] -= y1Rb * bx * xR;
  // x = 1 / ((s - sL*) (s - sR*))
  {
    const double qb = -xLb * xL * xL;
    sLb += qb * ((sL - sRs) + (sL - sLs));
    sLsb -= qb * (sL - sRs);
    sRsb -= qb * (sL - sLs);
  }
  {
    const double qb = -xRb * xR * xR;
    sRb += qb * ((sR - sRs) + (sR - sLs));
    sLsb -= qb * (sR - sRs);
    sRsb -= qb * (sR - sLs);
  }
  // sL* = u* - |bx| sqri, sR* = u* + |bx| sqri
  usb += sLsb + sRsb;
  sqrib += (sRsb - sLsb) * abx;
  bxb += (sRsb - sLsb) * sqri * sgn(bx);
  rhosib += sqrib * 0.5 / sqri;
  rhosb -= rhosib * rhosi * rhosi;
  // u* = frho* / rho*
  const double frhosb = usb / rhos;
  rhosb -= usb * us / rhos;
  // the averages: numerator / (sR - sL)
  const double Dib = rhosb * nr + mxsb * nm + frhosb * nf + pscsb * np;
  {
    const int ks[3] = {RHO, MX, PSC};
    const double bs[3] = {rhosb * Di, mxsb * Di, pscsb * Di};
    for (int q = 0; q < 3; ++q) {
      const int k = ks[q];
      const double b = bs[q];
      sRb += b * uR[k];
      uRb[k] += b * sR;
      sLb -= b * uL[k];
      uLb[k] -= b * sL;
      fRb[k] -= b;
      fLb[k] += b;
    }
  }
  {
    const double b = frhosb * Di;
    sRb += b * (fL[RHO] + sL * (uR[RHO] - uL[RHO]));
    sLb += b * (-fR[RHO] + sR * (uR[RHO] - uL[RHO]));
    fLb[RHO] += b * sR;
    fRb[RHO] -= b * sL;
    uRb[RHO] += b * sR * sL;
    uLb[RHO] -= b * sR * sL;
  }
  const double Db = -Dib * Di * Di;
  sRb += Db;
  sLb -= Db;
  wLb[BX] += bxb;
  vjp_flux(wL, fLb, gam, wLb);
  vjp_flux(wR, fRb, gam, wRb);
  vjp_prim2cons(wL, uLb, gam, wLb);
  vjp_prim2cons(wR, uRb, gam, wRb);
  vjp_wave_speeds(wL, wR, cfL, cfR, gam, sLb, sRb, wLb, wRb);
}

// HLLD flux (fluxes_c.c:616-834, as restated in bnz_device.cuh flux_hlld):
// given fb, add wLb, wRb (the normal field's cotangent is split over the BX
// entries of both sides; the caller sums them).  The fan region is the one
// the forward selects for these states.
BNZ_HD void vjp_hlld(const double* wL, const double* wR, double gam, const double* fb, double* wLb, double* wRb) {
  // ---- forward (values kept for the reverse sweep) ----
  const double bx = wL[BX];
  const double bx2 = sq(bx);
  const double rL = wL[RHO], rR = wR[RHO];
  const double vxL = wL[VX], vxR = wR[VX];
  const double b2L = bx2 + sq(wL[BY]) + sq(wL[BZ]);
  const double b2R = bx2 + sq(wR[BY]) + sq(wR[BZ]);
  const double ptL = wL[PR] + 0.5 * b2L, ptR = wR[PR] + 0.5 * b2R;
  const double mxL = rL * vxL, mxR = rR * vxR;
  const double fmxL = mxL * vxL + ptL - bx2, fmxR = mxR * vxR + ptR - bx2;
  const double cfL = fms_val(wL, gam), cfR = fms_val(wR, gam);
  const double cfm = cfL > cfR ? cfL : cfR;
  const double sL = (vxL < vxR ? vxL : vxR) - cfm;
  const double sR = (vxL > vxR ? vxL : vxR) + cfm;
  const double den = sR * rR - sL * rL - (mxR - mxL);
  const double deni = quo(1., den);
  const double num = sR * mxR - sL * mxL - (fmxR - fmxL);
  const double sM = num * deni;
  const double sLvxL = sL - vxL, sRvxR = sR - vxR;
#if BNZ_FAST_MATH && defined(__CUDA_ARCH__)
  // the fast forward's forms (bnz_device.cuh flux_hlld): one division for both
  const double dLM = sL - sM, dRM = sR - sM;
  const double inv2 = quo(1., dLM * dRM);
  const double sLsMi = dRM * inv2, sRsMi = dLM * inv2;
#else
  const double sLsMi = 1. / (sL - sM), sRsMi = 1. / (sR - sM);
#endif
  const double xL = sLvxL * sLsMi, xR = sRvxR * sRsMi;
  const double rLs = rL * xL, rRs = rR * xR;
  const double pts = rL * sLvxL * (sM - vxL) + ptL;
  const double rvL = rL * sLvxL, rvR = rR * sRvxR;
#if BNZ_FAST_MATH && defined(__CUDA_ARCH__)
  const double DL = rvL * (sL - sM) - bx2, DR = rvR * (sR - sM) - bx2;
  const double iD = quo(1., DL * DR);
  const double wvbL = DR * iD, wvbR = DL * iD;
#else
  const double wvbL = 1. / (rvL * (sL - sM) - bx2), wvbR = 1. / (rvR * (sR - sM) - bx2);
#endif
  const double wvL = bx * (sM - vxL) * wvbL, wvR = bx * (sM - vxR) * wvbR;
  const double vyLs = wL[VY] - wL[BY] * wvL, vyRs = wR[VY] - wR[BY] * wvR;
  const double vzLs = wL[VZ] - wL[BZ] * wvL, vzRs = wR[VZ] - wR[BZ] * wvR;
  const double QL = rvL * sLvxL - bx2, QR = rvR * sRvxR - bx2;
  const double wbL = QL * wvbL, wbR = QR * wvbR;
  const double byLs = wL[BY] * wbL, byRs = wR[BY] * wbR;
  const double bzLs = wL[BZ] * wbL, bzRs = wR[BZ] * wbR;
  const double vsbsL = sM * bx + vyLs * byLs + vzLs * bzLs;
  const double vsbsR = sM * bx + vyRs * byRs + vzRs * bzRs;
#if BNZ_FAST_MATH && defined(__CUDA_ARCH__)
  const double isrL = rsqrt(rLs), isrR = rsqrt(rRs);
  const double srL = rLs * isrL, srR = rRs * isrR;
#else
  const double srL = sqrt(rLs), srR = sqrt(rRs);
  const double isrL = 1. / srL, isrR = 1. / srR;
#endif
  const double abx = fabs(bx);
  const double sLs = sM - abx * isrL, sRs = sM + abx * isrR;
  int r = 0;
  if (sL > 0.) r = 1;
  if (sL <= 0. && 0. < sLs) r = 2;
  if (sLs <= 0. && 0. < sM) r = 3;
  if (sM <= 0. && 0. < sRs) r = 4;
  if (sRs <= 0. && 0. < sR) r = 5;
  if (sR <= 0.) r = 6;
  if (r == 0) return;
  const double dsum = srL + srR;
  const double rhoLRi = quo(1., dsum);
  const double sgnb = sgn(bx);
  const double Nvy = srL * vyLs + srR * vyRs + (byRs - byLs) * sgnb;
  const double Nvz = srL * vzLs + srR * vzRs + (bzRs - bzLs) * sgnb;
  const double Nby = srL * byRs + srR * byLs + srL * srR * (vyRs - vyLs) * sgnb;
  const double Nbz = srL * bzRs + srR * bzLs + srL * srR * (vzRs - vzLs) * sgnb;
  const double vyss = Nvy * rhoLRi, vzss = Nvz * rhoLRi;
  const double byss = Nby * rhoLRi, bzss = Nbz * rhoLRi;
  const double vssbss = sM * bx + vyss * byss + vzss * bzss;

  const bool left = r <= 3;
  const double* w = left ? wL : wR;
  double* wb = left ? wLb : wRb;
  const double s_o = left ? sL : sR;
  const double s_i = left ? sLs : sRs;
  const double x = left ? xL : xR;
  const double svx = left ? sLvxL : sRvxR;
  const double sMi = left ? sLsMi : sRsMi;
  const double pt = left ? ptL : ptR;
  const double rs = left ? rLs : rRs;
  const double vys = left ? vyLs : vyRs, vzs = left ? vzLs : vzRs;
  const double bys = left ? byLs : byRs, bzs = left ? bzLs : bzRs;
  const double vsbs = left ? vsbsL : vsbsR;
  const double srs = left ? srL : srR;
  double u[NM], f[NM];
  cons_of(w, gam, u);
  flux_of(w, gam, f);
  const double dotvb = w[VX] * bx + w[VY] * w[BY] + w[VZ] * w[BZ];
  const double nume = svx * u[EN] - pt * w[VX] + pts * sM + bx * (dotvb - vsbs);
  const double es = nume * sMi;
  const double us[NM] = {rs, rs * sM, rs * vys, rs * vzs, es, u[PSC] * x, 0., bys, bzs};
  const double t = srs * (vsbs - vssbss) * sgnb;
  const double ess = left ? es - t : es + t;
  const double uss[NM] = {rs, rs * sM, rs * vyss, rs * vzss, ess, u[PSC] * x, 0., byss, bzss};

  // ---- reverse ----
  double F[NM];
  for (int n = 0; n < NM; ++n) F[n] = n == BX ? 0. : fb[n];
  double fbb[NM], ub[NM], usb[NM], ussb[NM];
  double s_ob = 0., s_ib = 0.;
  for (int n = 0; n < NM; ++n) {
    fbb[n] = F[n];
    ub[n] = 0.;
    usb[n] = 0.;
    ussb[n] = 0.;
  }
  if (r == 2 || r == 5 || r == 3 || r == 4) {
    for (int n = 0; n < NM; ++n) {
      s_ob += F[n] * (us[n] - u[n]);
      usb[n] += s_o * F[n];
      ub[n] -= s_o * F[n];
    }
  }
  if (r == 3 || r == 4) {
    for (int n = 0; n < NM; ++n) {
      s_ib += F[n] * (uss[n] - us[n]);
      ussb[n] += s_i * F[n];
      usb[n] -= s_i * F[n];
    }
  }
  // scalar cotangents
  double rsb = 0., sMb = 0., vyssb = 0., vzssb = 0., essb = 0., xb = 0., byssb = 0., bzssb = 0.;
  double vysb = 0., vzsb = 0., esb = 0., bysb = 0., bzsb = 0.;
  double uPSCb = 0.;
  // uss
  rsb += ussb[0] + ussb[1] * sM + ussb[2] * vyss + ussb[3] * vzss;
  sMb += ussb[1] * rs;
  vyssb += ussb[2] * rs;
  vzssb += ussb[3] * rs;
  essb += ussb[4];
  uPSCb += ussb[5] * x;
  xb += ussb[5] * u[PSC];
  byssb += ussb[7];
  bzssb += ussb[8];
  // ess = es -+ t ; t = srs (vsbs - vssbss) sgnb
  esb += essb;
  const double tb = left ? -essb : essb;
  double srsb = tb * (vsbs - vssbss) * sgnb;
  double vsbsb = tb * srs * sgnb;
  double vssbssb = -tb * srs * sgnb;
  // us
  rsb += usb[0] + usb[1] * sM + usb[2] * vys + usb[3] * vzs;
  sMb += usb[1] * rs;
  vysb += usb[2] * rs;
  vzsb += usb[3] * rs;
  esb += usb[4];
  uPSCb += usb[5] * x;
  xb += usb[5] * u[PSC];
  bysb += usb[7];
  bzsb += usb[8];
  // es = nume * sMi
  const double numeb = esb * sMi;
  double sMib = esb * nume;
  double svxb = numeb * u[EN];
  ub[EN] += numeb * svx;
  double ptb = -numeb * w[VX];
  wb[VX] -= numeb * pt;
  double ptsb = numeb * sM;
  sMb += numeb * pts;
  double bxb = numeb * (dotvb - vsbs);
  vsbsb -= numeb * bx;
  {
    const double db = numeb * bx;
    wb[VX] += db * bx;
    bxb += db * w[VX];
    wb[VY] += db * w[BY];
    wb[BY] += db * w[VY];
    wb[VZ] += db * w[BZ];
    wb[BZ] += db * w[VZ];
  }
  ub[PSC] += uPSCb;
  // u and f of the side (u = prim2cons(w), f = flux(w))
  vjp_flux(w, fbb, gam, wb);
  vjp_prim2cons(w, ub, gam, wb);
  // vssbss = sM bx + vyss byss + vzss bzss
  sMb += vssbssb * bx;
  bxb += vssbssb * sM;
  vyssb += vssbssb * byss;
  byssb += vssbssb * vyss;
  vzssb += vssbssb * bzss;
  bzssb += vssbssb * vzss;
  // double-star tangential state
  double srLb = 0., srRb = 0., rhoLRib = 0.;
  double vyLsb = 0., vyRsb = 0., vzLsb = 0., vzRsb = 0., byLsb = 0., byRsb = 0., bzLsb = 0., bzRsb = 0.;
  {
    const double Nb = byssb * rhoLRi;
    rhoLRib += byssb * Nby;
    srLb += Nb * (byRs + srR * (vyRs - vyLs) * sgnb);
    srRb += Nb * (byLs + srL * (vyRs - vyLs) * sgnb);
    byRsb += Nb * srL;
    byLsb += Nb * srR;
    vyRsb += Nb * srL * srR * sgnb;
    vyLsb -= Nb * srL * srR * sgnb;
  }
  {
    const double Nb = bzssb * rhoLRi;
    rhoLRib += bzssb * Nbz;
    srLb += Nb * (bzRs + srR * (vzRs - vzLs) * sgnb);
    srRb += Nb * (bzLs + srL * (vzRs - vzLs) * sgnb);
    bzRsb += Nb * srL;
    bzLsb += Nb * srR;
    vzRsb += Nb * srL * srR * sgnb;
    vzLsb -= Nb * srL * srR * sgnb;
  }
  {
    const double Nb = vyssb * rhoLRi;
    rhoLRib += vyssb * Nvy;
    srLb += Nb * vyLs;
    vyLsb += Nb * srL;
    srRb += Nb * vyRs;
    vyRsb += Nb * srR;
    byRsb += Nb * sgnb;
    byLsb -= Nb * sgnb;
  }
  {
    const double Nb = vzssb * rhoLRi;
    rhoLRib += vzssb * Nvz;
    srLb += Nb * vzLs;
    vzLsb += Nb * srL;
    srRb += Nb * vzRs;
    vzRsb += Nb * srR;
    bzRsb += Nb * sgnb;
    bzLsb -= Nb * sgnb;
  }
  {
    const double db = -rhoLRib * rhoLRi * rhoLRi;
    srLb += db;
    srRb += db;
  }
  // side selections (one side's copies of the scalar star quantities)
  double sLb = 0., sRb = 0., sLsb = 0., sRsb = 0., xLb = 0., xRb = 0., sLvxLb = 0., sRvxRb = 0.;
  double sLsMib = 0., sRsMib = 0., ptLb = 0., ptRb = 0., rLsb = 0., rRsb = 0.;
  if (left) {
    sLb += s_ob;
    sLsb += s_ib;
    xLb += xb;
    sLvxLb += svxb;
    sLsMib += sMib;
    ptLb += ptb;
    rLsb += rsb;
    vyLsb += vysb;
    vzLsb += vzsb;
    byLsb += bysb;
    bzLsb += bzsb;
    srLb += srsb;
  } else {
    sRb += s_ob;
    sRsb += s_ib;
    xRb += xb;
    sRvxRb += svxb;
    sRsMib += sMib;
    ptRb += ptb;
    rRsb += rsb;
    vyRsb += vysb;
    vzRsb += vzsb;
    byRsb += bysb;
    bzRsb += bzsb;
    srRb += srsb;
  }
  // vsbs (the chosen side's copy) and pts
  double vsbsLb = left ? vsbsb : 0., vsbsRb = left ? 0. : vsbsb;
  // sLs = sM - |bx| / srL ; sRs = sM + |bx| / srR
  sMb += sLsb + sRsb;
  bxb += (-sLsb * isrL + sRsb * isrR) * sgn(bx);
  srLb += sLsb * abx * isrL * isrL;
  srRb -= sRsb * abx * isrR * isrR;
  // srL = sqrt(rLs)
  rLsb += srLb * 0.5 * isrL;
  rRsb += srRb * 0.5 * isrR;
  // vsbs = sM bx + vys bys + vzs bzs (both sides)
  sMb += (vsbsLb + vsbsRb) * bx;
  bxb += (vsbsLb + vsbsRb) * sM;
  vyLsb += vsbsLb * byLs;
  byLsb += vsbsLb * vyLs;
  vzLsb += vsbsLb * bzLs;
  bzLsb += vsbsLb * vzLs;
  vyRsb += vsbsRb * byRs;
  byRsb += vsbsRb * vyRs;
  vzRsb += vsbsRb * bzRs;
  bzRsb += vsbsRb * vzRs;
  // bys = by wb
  double wbLb = byLsb * wL[BY] + bzLsb * wL[BZ];
  double wbRb = byRsb * wR[BY] + bzRsb * wR[BZ];
  wLb[BY] += byLsb * wbL;
  wLb[BZ] += bzLsb * wbL;
  wRb[BY] += byRsb * wbR;
  wRb[BZ] += bzRsb * wbR;
  // wb = Q wvb
  double wvbLb = wbLb * QL, wvbRb = wbRb * QR;
  const double QLb = wbLb * wvbL, QRb = wbRb * wvbR;
  double rvLb = QLb * sLvxL, rvRb = QRb * sRvxR;
  sLvxLb += QLb * rvL;
  sRvxRb += QRb * rvR;
  double bx2b = -QLb - QRb;
  // vys = vy - by wv ; vzs = vz - bz wv
  wLb[VY] += vyLsb;
  wLb[VZ] += vzLsb;
  wRb[VY] += vyRsb;
  wRb[VZ] += vzRsb;
  wLb[BY] -= vyLsb * wvL;
  wLb[BZ] -= vzLsb * wvL;
  wRb[BY] -= vyRsb * wvR;
  wRb[BZ] -= vzRsb * wvR;
  const double wvLb = -vyLsb * wL[BY] - vzLsb * wL[BZ];
  const double wvRb = -vyRsb * wR[BY] - vzRsb * wR[BZ];
  // wv = bx (sM - vx) wvb
  bxb += wvLb * (sM - vxL) * wvbL + wvRb * (sM - vxR) * wvbR;
  sMb += wvLb * bx * wvbL + wvRb * bx * wvbR;
  wLb[VX] -= wvLb * bx * wvbL;
  wRb[VX] -= wvRb * bx * wvbR;
  wvbLb += wvLb * bx * (sM - vxL);
  wvbRb += wvRb * bx * (sM - vxR);
  // wvb = 1 / (rv (s - sM) - bx2)
  {
    const double DLb = -wvbLb * wvbL * wvbL, DRb = -wvbRb * wvbR * wvbR;
    rvLb += DLb * (sL - sM);
    sLb += DLb * rvL;
    sMb -= DLb * rvL;
    bx2b -= DLb;
    rvRb += DRb * (sR - sM);
    sRb += DRb * rvR;
    sMb -= DRb * rvR;
    bx2b -= DRb;
  }
  // rv = rho (s - vx)
  double rLb = rvLb * sLvxL, rRb = rvRb * sRvxR;
  sLvxLb += rvLb * rL;
  sRvxRb += rvRb * rR;
  // pts = rL sLvxL (sM - vxL) + ptL
  rLb += ptsb * sLvxL * (sM - vxL);
  sLvxLb += ptsb * rL * (sM - vxL);
  sMb += ptsb * rL * sLvxL;
  wLb[VX] -= ptsb * rL * sLvxL;
  ptLb += ptsb;
  // rs = rho x
  rLb += rLsb * xL;
  xLb += rLsb * rL;
  rRb += rRsb * xR;
  xRb += rRsb * rR;
  // x = svx sMi
  sLvxLb += xLb * sLsMi;
  sLsMib += xLb * sLvxL;
  sRvxRb += xRb * sRsMi;
  sRsMib += xRb * sRvxR;
  // sMi = 1 / (s - sM)
  {
    const double eL = -sLsMib * sLsMi * sLsMi, eR = -sRsMib * sRsMi * sRsMi;
    sLb += eL;
    sMb -= eL;
    sRb += eR;
    sMb -= eR;
  }
  // svx = s - vx
  sLb += sLvxLb;
  wLb[VX] -= sLvxLb;
  sRb += sRvxRb;
  wRb[VX] -= sRvxRb;
  // sM = num deni ; deni = 1 / den
  const double numb = sMb * deni;
  const double denb = -sMb * num * deni * deni;
  // num = sR mxR - sL mxL - (fmxR - fmxL)
  sRb += numb * mxR;
  double mxRb = numb * sR;
  sLb -= numb * mxL;
  double mxLb = -numb * sL;
  const double fmxRb = -numb, fmxLb = numb;
  // den = sR rR - sL rL - (mxR - mxL)
  sRb += denb * rR;
  rRb += denb * sR;
  sLb -= denb * rL;
  rLb -= denb * sL;
  mxRb -= denb;
  mxLb += denb;
  // fmx = mx vx + pt - bx2
  mxLb += fmxLb * vxL;
  wLb[VX] += fmxLb * mxL;
  ptLb += fmxLb;
  mxRb += fmxRb * vxR;
  wRb[VX] += fmxRb * mxR;
  ptRb += fmxRb;
  bx2b -= fmxLb + fmxRb;
  // mx = rho vx
  rLb += mxLb * vxL;
  wLb[VX] += mxLb * rL;
  rRb += mxRb * vxR;
  wRb[VX] += mxRb * rR;
  // pt = p + 0.5 b2 ; b2 = bx2 + by^2 + bz^2
  wLb[PR] += ptLb;
  wRb[PR] += ptRb;
  bx2b += 0.5 * (ptLb + ptRb);
  wLb[BY] += ptLb * wL[BY];
  wLb[BZ] += ptLb * wL[BZ];
  wRb[BY] += ptRb * wR[BY];
  wRb[BZ] += ptRb * wR[BZ];
  wLb[RHO] += rLb;
  wRb[RHO] += rRb;
  // wave speeds
  vjp_wave_speeds(wL, wR, cfL, cfR, gam, sLb, sRb, wLb, wRb);
  // the normal field
  bxb += 2. * bx * bx2b;
  wLb[BX] += bxb;
}

// Slope limiters (reconstr_c.h:28-44): partial derivatives of lim(a, b).
template <int LIM>
BNZ_HD void lim_grad(double a, double b, double& da, double& db) {
  if (LIM == 2) {  // minmod
    da = db = 0.;
    if (a * b <= 0.) return;
    if (a > 0.) {
      if (a < b) da = 1.;
      else db = 1.;
    } else {
      if (a > b) da = 1.;
      else db = 1.;
    }
  } else if (LIM == 1) {  // mc: mm(2 mm(a, b), 0.5 (a + b))
    da = db = 0.;
    double m1a, m1b;
    lim_grad<2>(a, b, m1a, m1b);
    double m1;
    m1 = (a * b <= 0.) ? 0. : ((a > 0.) ? ((a < b) ? a : b) : ((a > b) ? a : b));
    const double p = 2. * m1, q = 0.5 * (a + b);
    double dp, dq;
    lim_grad<2>(p, q, dp, dq);
    da = dp * 2. * m1a + dq * 0.5;
    db = dp * 2. * m1b + dq * 0.5;
  } else {  // van Leer: 2ab / (a + b) for ab > 0
    const double ab = a * b;
    if (ab > 0.) {
      const double s = a + b;
      da = 2. * b * b / (s * s);
      db = 2. * a * a / (s * s);
    } else {
      da = db = 0.;
    }
  }
}

BNZ_HD void lim_grad_rt(int lim, double a, double b, double& da, double& db) {
  if (lim == 1) lim_grad<1>(a, b, da, db);
  else if (lim == 2) lim_grad<2>(a, b, da, db);
  else lim_grad<0>(a, b, da, db);
}

BNZ_HD double lim_val_rt(int lim, double a, double b) {
  const double ab = a * b;
  if (lim == 0) return ab > 0. ? 2. * ab / (a + b) : 0.;
  const double mm = ab <= 0. ? 0. : (a > 0. ? (a < b ? a : b) : (a > b ? a : b));
  if (lim == 2) return mm;
  const double p = 2. * mm, q = 0.5 * (a + b);
  return p * q <= 0. ? 0. : (p > 0. ? (p < q ? p : q) : (p > q ? p : q));
}

// ---- characteristic projection of the PLM slopes (charact_proj) ----------
// prim2char / char2prim of eos_c.h:100-333 as restated in bnz_device.cuh.
// Both are linear in the differences they map, with coefficients built from
// the cell state (rho, p and the three B components of the local frame).  The
// VJP applies their transposes column by column and differentiates the
// coefficients in forward mode: a Dual carries the derivative of every
// coefficient along one direction of the cell state, through the same square
// roots, divisions and case switches (taken on the values) as the forward.
struct Dual {
  double v, d;
  BNZ_HD Dual(double x = 0., double y = 0.) : v(x), d(y) {}
};
BNZ_HD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
BNZ_HD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
BNZ_HD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
BNZ_HD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
BNZ_HD Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
BNZ_HD double val(double x) { return x; }
BNZ_HD double val(Dual x) { return x.v; }
BNZ_HD double tsqrt(double x) { return sqrt(x); }
BNZ_HD Dual tsqrt(Dual x) {
  const double r = sqrt(x.v);
  return Dual(r, r > 0. ? 0.5 * x.d / r : 0.);
}
BNZ_HD double tabs(double x) { return fabs(x); }
BNZ_HD Dual tabs(Dual x) { return x.v >= 0. ? x : -x; }

template <class T>
struct CharK {
  T rho, rhoi, a2rho, a, cf, cs, af, as, betay, betaz;
  double s;
};

template <class T>
BNZ_HD void char_basis(T rho, T p, T bx, T by, T bz, double gam, CharK<T>& k) {
  k.rho = rho;
  k.rhoi = T(1.) / rho;
  k.s = sgn(val(bx));
  k.a2rho = T(gam) * p;
  k.a = tsqrt(k.a2rho * k.rhoi);
  const T bx2 = bx * bx;
  const T bperp2 = by * by + bz * bz;
  const T x = k.a2rho + (bx2 + bperp2);
  const T y = tsqrt(tabs(x * x - T(4.) * k.a2rho * bx2));
  const T cf2 = T(0.5) * (x + y), cs2 = T(0.5) * (x - y);
  k.cf = tsqrt(k.rhoi * cf2);
  k.cs = tsqrt(k.rhoi * tabs(cs2));
  if (val(k.cf) <= val(k.cs)) {
    k.af = T(1.);
    k.as = T(0.);
  } else if (val(k.a) <= val(k.cs)) {
    k.af = T(0.);
    k.as = T(1.);
  } else if (val(k.cf) <= val(k.a)) {
    k.af = T(1.);
    k.as = T(0.);
  } else {
    const T z = T(1.) / (cf2 - cs2);
    k.af = tsqrt(z * tabs(k.a2rho - cs2));
    k.as = tsqrt(z * tabs(cf2 - k.a2rho));
  }
  if (val(bperp2) != 0.) {
    const T bperpi = T(1.) / tsqrt(bperp2);
    k.betay = bperpi * by;
    k.betaz = bperpi * bz;
  } else {
    k.betay = T(0.);
    k.betaz = T(0.);
  }
}

// out = prim2char(d); PSC and BX pass through
template <class T>
BNZ_HD void p2c_apply(const CharK<T>& k, const T* d, T* out) {
  const T s = T(k.s);
  const T nf = T(0.5) / (k.a2rho * k.rhoi);
  const T qf_ = nf * k.cf * k.af * s, qs_ = nf * k.cs * k.as * s;
  const T af_ = nf * k.af, as_ = nf * k.as;
  const T rhoisr = tsqrt(k.rhoi);
  const T arhoisr = k.a * rhoisr;
  const T Af_ = af_ * arhoisr, As_ = as_ * arhoisr;
  const T x = s * rhoisr;
  const T v = k.betay * d[VY] + k.betaz * d[VZ];
  const T b = k.betay * d[BY] + k.betaz * d[BZ];
  const T tb = -(k.betaz * d[BY]) + k.betay * d[BZ];
  out[RHO] = af_ * (k.rhoi * d[PR] - k.cf * d[VX]) + qs_ * v + As_ * b;
  out[VX] = T(0.5) * ((-(k.betaz * d[VY]) + k.betay * d[VZ]) + x * tb);
  out[VY] = as_ * (k.rhoi * d[PR] - k.cs * d[VX]) - qf_ * v - Af_ * b;
  out[VZ] = d[RHO] - T(2.) * nf * d[PR];
  out[PR] = as_ * (k.rhoi * d[PR] + k.cs * d[VX]) + qf_ * v - Af_ * b;
  out[PSC] = d[PSC];
  out[BX] = d[BX];
  out[BY] = T(0.5) * ((k.betaz * d[VY] - k.betay * d[VZ]) + x * tb);
  out[BZ] = af_ * (k.rhoi * d[PR] + k.cf * d[VX]) - qs_ * v + As_ * b;
}

// out = char2prim(c); PSC and BX pass through
template <class T>
BNZ_HD void c2p_apply(const CharK<T>& k, const T* c, T* out) {
  const T s = T(k.s);
  const T qf = k.cf * k.af * s, qs = k.cs * k.as * s;
  const T rhosr = tsqrt(k.rho);
  const T arhosr = k.a * rhosr;
  const T Af = k.af * arhosr, As = k.as * arhosr;
  const T fa = k.af * (c[RHO] + c[BZ]) + k.as * (c[VY] + c[PR]);
  const T t = qs * (c[RHO] - c[BZ]) - qf * (c[VY] - c[PR]);
  const T u = As * (c[RHO] + c[BZ]) - Af * (c[VY] + c[PR]);
  const T srs = s * rhosr;
  out[RHO] = k.rho * fa + c[VZ];
  out[VX] = k.cf * k.af * (c[BZ] - c[RHO]) + k.cs * k.as * (c[PR] - c[VY]);
  out[VY] = k.betay * t - k.betaz * (c[VX] - c[BY]);
  out[VZ] = k.betaz * t + k.betay * (c[VX] - c[BY]);
  out[PR] = k.a2rho * fa;
  out[PSC] = c[PSC];
  out[BX] = c[BX];
  out[BY] = k.betay * u - k.betaz * srs * (c[VX] + c[BY]);
  out[BZ] = k.betaz * u + k.betay * srs * (c[VX] + c[BY]);
}

// d = half_slopes_char(wm, wc, wp) (reconstr_c.c:54-91 with charact_proj):
// the projected, limited and halved slope of the cell wc, local frame.
BNZ_HD void slopes_char(int lim, const double* wm, const double* wc, const double* wp, double gam, double* d) {
  CharK<double> k;
  char_basis<double>(wc[RHO], wc[PR], wc[BX], wc[BY], wc[BZ], gam, k);
  double dm0[NM], dp0[NM], dm[NM], dp[NM], c[NM];
  for (int n = 0; n < NM; ++n) {
    dm0[n] = wc[n] - wm[n];
    dp0[n] = wp[n] - wc[n];
  }
  p2c_apply<double>(k, dm0, dm);
  p2c_apply<double>(k, dp0, dp);
  for (int n = 0; n < NM; ++n) c[n] = 0.5 * lim_val_rt(lim, dm[n], dp[n]);
  c2p_apply<double>(k, c, d);
}

// VJP of slopes_char: given db (9), add the cotangents of wm, wc, wp.
BNZ_HD void vjp_slopes_char(int lim, const double* wm, const double* wc, const double* wp, double gam,
                            const double* db, double* wmb, double* wcb, double* wpb) {
  CharK<double> k;
  char_basis<double>(wc[RHO], wc[PR], wc[BX], wc[BY], wc[BZ], gam, k);
  double dm0[NM], dp0[NM], dm[NM], dp[NM], c[NM];
  for (int n = 0; n < NM; ++n) {
    dm0[n] = wc[n] - wm[n];
    dp0[n] = wp[n] - wc[n];
  }
  p2c_apply<double>(k, dm0, dm);
  p2c_apply<double>(k, dp0, dp);
  for (int n = 0; n < NM; ++n) c[n] = 0.5 * lim_val_rt(lim, dm[n], dp[n]);
  // cb = Q^T db, then through the limiter, then dm0b = P^T dmb (columns of
  // Q and P are their applications to unit vectors)
  double e[NM], col[NM], cb[NM], dmb[NM], dpb[NM];
  for (int q = 0; q < NM; ++q) {
    for (int n = 0; n < NM; ++n) e[n] = n == q ? 1. : 0.;
    c2p_apply<double>(k, e, col);
    double acc = 0.;
    for (int n = 0; n < NM; ++n) acc += db[n] * col[n];
    cb[q] = acc;
  }
  for (int n = 0; n < NM; ++n) {
    double la, lb;
    lim_grad_rt(lim, dm[n], dp[n], la, lb);
    dmb[n] = 0.5 * cb[n] * la;
    dpb[n] = 0.5 * cb[n] * lb;
  }
  for (int q = 0; q < NM; ++q) {
    for (int n = 0; n < NM; ++n) e[n] = n == q ? 1. : 0.;
    p2c_apply<double>(k, e, col);
    double am = 0., ap = 0.;
    for (int n = 0; n < NM; ++n) {
      am += dmb[n] * col[n];
      ap += dpb[n] * col[n];
    }
    wmb[q] -= am;
    wcb[q] += am - ap;
    wpb[q] += ap;
  }
  // the coefficients' dependence on wc, one state direction at a time
  const int ent[5] = {RHO, PR, BX, BY, BZ};
  for (int q = 0; q < 5; ++q) {
    Dual w5[5] = {Dual(wc[RHO]), Dual(wc[PR]), Dual(wc[BX]), Dual(wc[BY]), Dual(wc[BZ])};
    w5[q].d = 1.;
    CharK<Dual> kd;
    char_basis<Dual>(w5[0], w5[1], w5[2], w5[3], w5[4], gam, kd);
    Dual x[NM], y[NM];
    double phi = 0.;
    for (int n = 0; n < NM; ++n) x[n] = Dual(c[n]);
    c2p_apply<Dual>(kd, x, y);
    for (int n = 0; n < NM; ++n) phi += db[n] * y[n].d;
    for (int n = 0; n < NM; ++n) x[n] = Dual(dm0[n]);
    p2c_apply<Dual>(kd, x, y);
    for (int n = 0; n < NM; ++n) phi += dmb[n] * y[n].d;
    for (int n = 0; n < NM; ++n) x[n] = Dual(dp0[n]);
    p2c_apply<Dual>(kd, x, y);
    for (int n = 0; n < NM; ++n) phi += dpb[n] * y[n].d;
    wcb[ent[q]] += phi;
  }
}

// PLM face states of one variable at a face (reconstr_c.c:54-91):
//   wL = wm1 + 0.5 lim(wm1 - wm2, w0 - wm1),  wR = w0 - 0.5 lim(w0 - wm1, wp1 - w0).
// Given wLb, wRb, return the cotangents of (wm2, wm1, w0, wp1) in c[0..3].
BNZ_HD void vjp_plm(int lim, double wm2, double wm1, double w0, double wp1, double wLb, double wRb, double* c) {
  double la, lb;
  lim_grad_rt(lim, wm1 - wm2, w0 - wm1, la, lb);
  // wL
  c[0] = -0.5 * la * wLb;
  c[1] = wLb * (1. + 0.5 * la - 0.5 * lb);
  c[2] = 0.5 * lb * wLb;
  double ra, rb;
  lim_grad_rt(lim, w0 - wm1, wp1 - w0, ra, rb);
  // wR
  c[1] += 0.5 * ra * wRb;
  c[2] += wRb * (1. - 0.5 * ra + 0.5 * rb);
  c[3] = -0.5 * rb * wRb;
  c[0] += 0.;
}

}  // namespace adj
