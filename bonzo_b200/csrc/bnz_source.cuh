// bnz_source.cuh -- the source terms of the VL2 stages (src/srcterms):
// constant gravity (gravity.pyx:54-69) and the solenoidal driving force
// (turb_driv.pyx:34-124, turb_driv_c.c:5-95), applied after the flux and CT
// update of each stage (integrator.pyx:132-170 add_source_terms), before
// cons2prim.  gravity.pyx's constant-g loop reads a `u0` that is not in scope;
// the density and momentum of the stage input w0 are used, as the driving
// term does.  Included inside the per-floating-point-mode namespace.
#pragma once

namespace srcterm {

using namespace dev;

// u += dt (rho g, rho v.g) then u += dt (f, f.v), in the reference's order
__device__ __forceinline__ void apply(double* u, double rho, double vx, double vy, double vz, const double* g,
                                      bool grav, const double* f, double dt) {
  if (grav) {
    u[MX] += rho * g[0] * dt;
    u[MY] += rho * g[1] * dt;
    u[MZ] += rho * g[2] * dt;
    u[EN] += dt * ((rho * vx) * g[0] + (rho * vy) * g[1] + (rho * vz) * g[2]);
  }
  if (f) {
    u[MX] = u[MX] + dt * f[0];
    u[MY] = u[MY] + dt * f[1];
    u[MZ] = u[MZ] + dt * f[2];
    u[EN] = u[EN] + (dt * (f[0] * vx + f[1] * vy + f[2] * vz));
  }
}

// plain path: u1 on the stage's update box, w0 the stage input prim
__global__ void k_source(GridDev g, double* __restrict__ u1, const double* __restrict__ w0,
                         const double* __restrict__ fdriv, double gx, double gy, double gz, plain::Box box,
                         const double* dtp, double fac) {
  const double dt = fac * *dtp;
  const double gv[3] = {gx, gy, gz};
  const bool grav = gx != 0. || gy != 0. || gz != 0.;
  BOX_LOOP(box, i, j, k) {
    const long long c = plain::cidx(g, i, j, k);
    double u[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) u[n] = u1[n * g.sv + c];
    double f[3];
    if (fdriv) {
      f[0] = fdriv[c];
      f[1] = fdriv[g.sv + c];
      f[2] = fdriv[2 * g.sv + c];
    }
    apply(u, w0[c], w0[VX * g.sv + c], w0[VY * g.sv + c], w0[VZ * g.sv + c], gv, grav, fdriv ? f : nullptr, dt);
#pragma unroll
    for (int n = MX; n <= EN; ++n) u1[n * g.sv + c] = u[n];
  }
}

// turb_driv_c.c:5-95 at every cell of `box`: the curl of the mode sum at the
// cell centre, phases advanced by the reference's trigonometric recurrences,
// then the Ornstein-Uhlenbeck update f = (1 - dt/tau) f + sqrt(dt/tau) f0 g.
// modes = c1 then c2 (3 (2 nmod + 1)^3 each, turb_driv.pyx:50-79).
__global__ void k_drive(GridDev g, double* __restrict__ fdriv, const double* __restrict__ modes, int nmod,
                        double kx0, double ky0, double kz0, double tau, double f0, plain::Box box,
                        const double* dtp) {
  const double dt_tau = *dtp / tau;
  const double f1 = sqrt(dt_tau) * f0;
  const int nmod2 = 2 * nmod + 1;
  const double* c1 = modes;
  const double* c2 = modes + 3 * nmod2 * nmod2 * nmod2;
  const double nmodf = (double)nmod;
  BOX_LOOP(box, i, j, k) {
    const double x = g.lv[0][i], y = g.lv[1][j], z = g.lv[2][k];
    double th = -nmodf * (kx0 * x + ky0 * y + kz0 * z);
    double cn = cos(th), sn = sin(th);
    const double cnx = cos(kx0 * x), cny = cos(ky0 * y), cnz = cos(kz0 * z);
    const double snx = sin(kx0 * x), sny = sin(ky0 * y), snz = sin(kz0 * z);
    double gx = 0., gy = 0., gz = 0.;
    double tz = -nmodf * kz0;
    for (int p = 0; p < nmod2; ++p) {
      double ty = -nmodf * ky0;
      const double cn00 = cn, sn00 = sn;
      for (int q = 0; q < nmod2; ++q) {
        double tx = -nmodf * kx0;
        const double cn0 = cn, sn0 = sn;
        for (int r = 0; r < nmod2; ++r) {
          const int m = 3 * (r + nmod2 * q + nmod2 * nmod2 * p);
          const double ax = -c1[m] * sn + c2[m] * cn;
          const double ay = -c1[m + 1] * sn + c2[m + 1] * cn;
          const double az = -c1[m + 2] * sn + c2[m + 2] * cn;
          gx += ty * az - tz * ay;
          gy += -tx * az + tz * ax;
          gz += tx * ay - ty * ax;
          tx += kx0;
          const double cn_ = cn;
          cn = cn_ * cnx - sn * snx;
          sn = sn * cnx + cn_ * snx;
        }
        ty += ky0;
        cn = cn0;
        sn = sn0;
        const double cn_ = cn;
        cn = cn_ * cny - sn * sny;
        sn = sn * cny + cn_ * sny;
      }
      tz += kz0;
      cn = cn00;
      sn = sn00;
      const double cn_ = cn;
      cn = cn_ * cnz - sn * snz;
      sn = sn * cnz + cn_ * snz;
    }
    const long long c = plain::cidx(g, i, j, k);
    fdriv[c] = (1. - dt_tau) * fdriv[c] + f1 * gx;
    fdriv[g.sv + c] = (1. - dt_tau) * fdriv[g.sv + c] + f1 * gy;
    fdriv[2 * g.sv + c] = (1. - dt_tau) * fdriv[2 * g.sv + c] + f1 * gz;
  }
}

}  // namespace srcterm
