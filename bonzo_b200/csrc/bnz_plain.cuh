// bnz_plain.cuh -- reference-structured kernels: one kernel per loop of the
// reference's Cython step, interface states and fluxes through HBM.
//
// This is the "plain one-instance-per-launch" path: it follows
// src/integration/{godunov,ct,new_dt}.pyx loop by loop (same index ranges),
// with one thread per interface / cell instead of one OpenMP thread per row.
// Included inside the per-floating-point-mode namespace.
#pragma once

namespace plain {

using namespace dev;

__device__ __forceinline__ long long cidx(const GridDev& g, int i, int j, int k) {
  return ((long long)k * g.ny + j) * g.nx + i;
}

// godunov.pyx:297-324: local (sweep) variable n -> global variable index.
template <int AX>
__host__ __device__ constexpr int perm(int n) {
  return AX == 0 ? n
         : AX == 1 ? (n == VX ? VY : n == VY ? VZ : n == VZ ? VX : n == BX ? BY : n == BY ? BZ : n == BZ ? BX : n)
                   : (n == VX ? VZ : n == VY ? VX : n == VZ ? VY : n == BX ? BZ : n == BY ? BX : n == BZ ? BY : n);
}

__device__ __forceinline__ double half_slope_rt(int lim, double wm, double wc, double wp) {
  if (lim == LIM_MC) return half_slope<LIM_MC>(wm, wc, wp);
  if (lim == LIM_MM) return half_slope<LIM_MM>(wm, wc, wp);
  return half_slope<LIM_VL>(wm, wc, wp);
}

__device__ __forceinline__ void half_slopes_char_rt(int lim, const double* wm, const double* wc, const double* wp,
                                                    double gam, double* d) {
  if (lim == LIM_MC) half_slopes_char<LIM_MC>(wm, wc, wp, gam, d);
  else if (lim == LIM_MM) half_slopes_char<LIM_MM>(wm, wc, wp, gam, d);
  else half_slopes_char<LIM_VL>(wm, wc, wp, gam, d);
}

// Index boxes walk their cells with 32-bit unsigned arithmetic: a grid that
// fits in device memory (at 66 doubles a cell or more for the paths that use
// boxes, 180 GB hold about 340 M cells) has fewer than 2^31 cells, and 64-bit
// division by a runtime divisor costs several times the 32-bit one.
struct Box {
  int3 lo, hi;
  __device__ __forceinline__ unsigned size() const {
    return (unsigned)(hi.x - lo.x + 1) * (unsigned)(hi.y - lo.y + 1) * (unsigned)(hi.z - lo.z + 1);
  }
  __device__ __forceinline__ void at(unsigned t, int& i, int& j, int& k) const {
    const unsigned nxr = hi.x - lo.x + 1, nyr = hi.y - lo.y + 1;
    const unsigned r = t / nxr, q = r / nyr;
    i = lo.x + (int)(t - r * nxr);
    j = lo.y + (int)(r - q * nyr);
    k = lo.z + (int)q;
  }
};

#define BOX_LOOP(box, i, j, k)                                                                   \
  for (unsigned _t = blockIdx.x * blockDim.x + threadIdx.x, _n = (box).size(); _t < _n;          \
       _t += gridDim.x * blockDim.x)                                                             \
    if (int i, j, k; (box).at(_t, i, j, k), true)

// godunov.pyx:84-207: Godunov flux on the AX faces of `box` (face index along
// AX = the cell on its right).  ORDER 0: donor cell (reconstr_c.c:8-22);
// ORDER 1: PLM (reconstr_c.c:29-91).  Normal field from the face array.
// cp = 1 (charact_proj): the slopes are limited in characteristic variables.
template <int AX, int ORDER, int RS>
__global__ void __launch_bounds__(128) k_flux(GridDev g, const double* __restrict__ w,
                                              const double* __restrict__ bf, double* __restrict__ F,
                                              Box box, int lim, int cp, unsigned* err) {
  const long long s = AX == 0 ? 1LL : AX == 1 ? (long long)g.nx : (long long)g.nx * g.ny;
  unsigned e = 0;
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    double wL[NM], wR[NM];
    if (ORDER == 1 && cp) {
      double c4[4][NM], dl[NM], dr[NM];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int n = 0; n < NM; ++n) c4[q][n] = w[perm<AX>(n) * g.sv + c + (q - 2) * s];
      half_slopes_char_rt(lim, c4[0], c4[1], c4[2], g.gam, dl);
      half_slopes_char_rt(lim, c4[1], c4[2], c4[3], g.gam, dr);
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        wL[n] = c4[1][n] + dl[n];
        wR[n] = c4[2][n] - dr[n];
      }
    } else {
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        if (n == BX) continue;
        const double* a = w + perm<AX>(n) * g.sv + c;
        if (ORDER == 0) {
          wL[n] = a[-s];
          wR[n] = a[0];
        } else {
          double wm2 = a[-2 * s], wm1 = a[-s], w0 = a[0], wp1 = a[s];
          wL[n] = wm1 + half_slope_rt(lim, wm2, wm1, w0);
          wR[n] = w0 - half_slope_rt(lim, wm1, w0, wp1);
        }
      }
    }
    const double bx = bf[AX * g.sv + c];
    wL[BX] = bx;
    wR[BX] = bx;
    double f[NM];
    riemann<RS, true>(f, wL, wR, g.gam, e);
#pragma unroll
    for (int n = 0; n < NM; ++n) F[perm<AX>(n) * g.sv + c] = f[n];
  }
  if (e) atomicOr(err, e);
}

// godunov.pyx:215-252 (Cartesian areas and volumes, cartesian.pyx:97-115)
__global__ void k_advance_hydro(GridDev g, double* u1, const double* u0, const double* __restrict__ fx,
                                const double* __restrict__ fy, const double* __restrict__ fz, Box box,
                                const double* dtp, double fac) {
  const double dt = fac * *dtp;
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    double vol = g.dlf[0][i] * g.dlf[1][j] * g.dlf[2][k];
    double dtdv = dt / vol;
    double dax = g.dlf[1][j] * g.dlf[2][k];
    double day = g.dlf[0][i] * g.dlf[2][k];
    double daz = g.dlf[0][i] * g.dlf[1][j];
    const long long sy = g.nx, sz = (long long)g.nx * g.ny;
#pragma unroll
    for (int n = 0; n < BX; ++n) {
      const long long o = n * g.sv + c;
      double v = u0[o] - dtdv * (dax * fx[o + 1] - dax * fx[o]);
      if (g.dims >= 2) v -= dtdv * (day * fy[o + sy] - day * fy[o]);
      if (g.dims >= 3) v -= dtdv * (daz * fz[o + sz] - daz * fz[o]);
      u1[o] = v;
    }
  }
}

// ct.pyx:128-148
__global__ void k_ec(GridDev g, const double* __restrict__ w, double* __restrict__ ec, Box box) {
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    double vx = w[VX * g.sv + c], vy = w[VY * g.sv + c], vz = w[VZ * g.sv + c];
    double bx = w[BX * g.sv + c], by = w[BY * g.sv + c], bz = w[BZ * g.sv + c];
    ec[c] = -(vy * bz - vz * by);
    ec[g.sv + c] = (vx * bz - vz * bx);
    ec[2 * g.sv + c] = -(vx * by - vy * bx);
  }
}

// ct.pyx:153-215 (interp_ee1)
__global__ void k_ee(GridDev g, const double* __restrict__ ec, const double* __restrict__ fx,
                     const double* __restrict__ fy, const double* __restrict__ fz, double* __restrict__ ee,
                     Box box) {
  const long long sv = g.sv, sy = g.nx, sz = (long long)g.nx * g.ny;
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    if (g.dims == 3) {
      ee[c] = (0.5 * (-fy[BZ * sv + c - sz] - fy[BZ * sv + c] + fz[BY * sv + c - sy] + fz[BY * sv + c]) -
               0.25 * (ec[c - sy] + ec[c] + ec[c - sz - sy] + ec[c - sz]));
      ee[sv + c] = (0.5 * (-fz[BX * sv + c - 1] - fz[BX * sv + c] + fx[BZ * sv + c - sz] + fx[BZ * sv + c]) -
                    0.25 * (ec[sv + c - 1] + ec[sv + c] + ec[sv + c - sz - 1] + ec[sv + c - sz]));
      ee[2 * sv + c] =
          (0.5 * (-fx[BY * sv + c - sy] - fx[BY * sv + c] + fy[BX * sv + c - 1] + fy[BX * sv + c]) -
           0.25 * (ec[2 * sv + c - 1] + ec[2 * sv + c] + ec[2 * sv + c - sy - 1] + ec[2 * sv + c - sy]));
    } else if (g.dims == 2) {
      ee[c] = -fy[BZ * sv + c];
      ee[sv + c] = fx[BZ * sv + c];
      ee[2 * sv + c] =
          (0.5 * (-fx[BY * sv + c - sy] - fx[BY * sv + c] + fy[BX * sv + c - 1] + fy[BX * sv + c]) -
           0.25 * (ec[2 * sv + c - 1] + ec[2 * sv + c] + ec[2 * sv + c - sy - 1] + ec[2 * sv + c - sy]));
    } else {
      ee[c] = -ec[c];
      ee[sv + c] = fx[BZ * sv + c];
      ee[2 * sv + c] = -fx[BY * sv + c];
    }
  }
}

// ct.pyx:15-91, one face component per launch (COMP = 0, 1, 2).
template <int COMP>
__global__ void k_advance_b(GridDev g, double* b1, const double* b0, const double* __restrict__ ee, Box box,
                            const double* dtp, double fac) {
  const double dt = fac * *dtp;
  const long long sv = g.sv, sy = g.nx, sz = (long long)g.nx * g.ny;
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    if (COMP == 0) {
      double dtda = dt / (g.dlf[1][j] * g.dlf[2][k]);
      double v = b0[c];
      if (g.dims >= 2) {
        double ds = g.dlf[2][k];
        v -= dtda * (ds * ee[2 * sv + c + sy] - ds * ee[2 * sv + c]);
      }
      if (g.dims >= 3) {
        double ds = g.dlf[1][j];
        v += dtda * (ds * ee[sv + c + sz] - ds * ee[sv + c]);
      }
      b1[c] = v;
    } else if (COMP == 1) {
      double dtda = dt / (g.dlf[0][i] * g.dlf[2][k]);
      double ds = g.dlf[2][k];
      double v = b0[sv + c] + dtda * (ds * ee[2 * sv + c + 1] - ds * ee[2 * sv + c]);
      if (g.dims >= 3) {
        double dsx = g.dlf[0][i];
        v -= dtda * (dsx * ee[c + sz] - dsx * ee[c]);
      }
      b1[sv + c] = v;
    } else {
      double dtda = dt / (g.dlf[0][i] * g.dlf[1][j]);
      double ds = g.dlf[1][j];
      double v = b0[2 * sv + c] - dtda * (ds * ee[sv + c + 1] - ds * ee[sv + c]);
      if (g.dims >= 2) {
        double dsx = g.dlf[0][i];
        v += dtda * (dsx * ee[c + sy] - dsx * ee[c]);
      }
      b1[2 * sv + c] = v;
    }
  }
}

// ct.pyx:96-123
__global__ void k_interp_bc(GridDev g, double* __restrict__ u, const double* __restrict__ b, Box box) {
  const long long sv = g.sv, sy = g.nx, sz = (long long)g.nx * g.ny;
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    u[BX * sv + c] = ((g.lv[0][i] - g.lf[0][i]) * b[c] + (g.lf[0][i + 1] - g.lv[0][i]) * b[c + 1]) * g.dlf_inv[0][i];
    if (g.dims >= 2)
      u[BY * sv + c] = ((g.lv[1][j] - g.lf[1][j]) * b[sv + c] + (g.lf[1][j + 1] - g.lv[1][j]) * b[sv + c + sy]) *
                       g.dlf_inv[1][j];
    else
      u[BY * sv + c] = b[sv + c];
    if (g.dims >= 3)
      u[BZ * sv + c] = ((g.lv[2][k] - g.lf[2][k]) * b[2 * sv + c] +
                        (g.lf[2][k + 1] - g.lv[2][k]) * b[2 * sv + c + sz]) * g.dlf_inv[2][k];
    else
      u[BZ * sv + c] = b[2 * sv + c];
  }
}

__device__ __forceinline__ unsigned check_prim(const double* w) {
  unsigned e = 0;
  if (!(w[RHO] > 0.)) e |= ERR_RHO;
  if (!(w[PR] > 0.)) e |= ERR_PRES;
  if (isnan(w[VX]) || isnan(w[VY]) || isnan(w[VZ]) || isnan(w[BX]) || isnan(w[BY]) || isnan(w[BZ])) e |= ERR_NAN;
  return e;
}

// eos.pyx:13-44 -> eos_c.c:9-26
__global__ void k_cons2prim(GridDev g, double* __restrict__ w, const double* __restrict__ u, Box box,
                            unsigned* err) {
  unsigned e = 0;
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    double uu[NM], ww[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) uu[n] = u[n * g.sv + c];
    cons2prim(ww, uu, g.gam);
    e |= check_prim(ww);
#pragma unroll
    for (int n = 0; n < NM; ++n) w[n * g.sv + c] = ww[n];
  }
  if (e) atomicOr(err, e);
}

// eos.pyx:48-78 -> eos_c.c:31-48
__global__ void k_prim2cons(GridDev g, double* __restrict__ u, const double* __restrict__ w, Box box) {
  BOX_LOOP(box, i, j, k) {
    const long long c = cidx(g, i, j, k);
    double uu[NM], ww[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) ww[n] = w[n * g.sv + c];
    prim2cons(uu, ww, g.gam);
#pragma unroll
    for (int n = 0; n < NM; ++n) u[n * g.sv + c] = uu[n];
  }
}

}  // namespace plain
