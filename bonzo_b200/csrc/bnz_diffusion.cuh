// bnz_diffusion.cuh -- RKL2 super-time-stepped electron thermal conduction.
//
// Follows src/dissipation/thcond_elec.pyx:17-466 and util_diffusion.pyx:16-159:
// temperature T = p/rho, harmonic-mean face conductivity, field-aligned face
// flux q = -kappa b (b . grad T) with limited transverse gradients (or the
// isotropic flux), optional saturation, dp/dt = -(gamma-1) div q, and the
// Meyer et al. (2014) RKL2 stage recursion (diffusion.pyx:217-260).
// Included inside the per-floating-point-mode namespace.
#pragma once

namespace diff {

using namespace dev;
constexpr double SMALL_NUM = 1.0e-20;

__device__ __forceinline__ long long c3(const GridDev& g, int i, int j, int k) {
  return ((long long)k * g.ny + j) * g.nx + i;
}

// util_diffusion.pyx:16-20 (returns a magnitude, as the reference does)
__device__ __forceinline__ double dlim(double a, double b) {
  double _a = fabs(a), _b = fabs(b);
  return fmax(0., fmin(fmin(0.5 * (_a + _b), _a), _b));
}

// thcond_elec.pyx:146-152 -- T = p / rho on every cell
__global__ void k_temp(GridDev g, const double* __restrict__ w, double* __restrict__ T) {
  const long long n = g.sv;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    T[c] = w[PR * g.sv + c] / w[RHO * g.sv + c];
}

__device__ __forceinline__ double saturate(double f, double h, double Tl, double Tr, double rl, double rr) {
  double Tc = 0.5 * (Tl + Tr);
  double rhoc = 0.5 * (rl + rr);
  double mom = 0.5 * h * rhoc * sqrt(0.67 * Tc);
  double qsat = f > 0. ? Tl * mom : Tr * mom;
  return f * qsat / (fabs(f) + qsat + SMALL_NUM);
}

// thcond_elec.pyx:154-303: the conductive flux through the AX face of cell
// (i, j, k) (the face between cells c - s and c), from T = p / rho.
template <int AX>
__device__ __forceinline__ double face_flux(const GridDev& g, const double* __restrict__ w,
                                            const double* __restrict__ bf, const double* __restrict__ T,
                                            const DiffArgs& da, int i, int j, int k) {
  const long long sy = g.nx, sz = (long long)g.nx * g.ny, sv = g.sv;
  const double k0 = da.kappa0;
  const double kappah = (2. * k0 * k0 / (k0 + k0 + SMALL_NUM));
  const double* dvi0 = g.dlv_inv[0];
  const double* dvi1 = g.dlv_inv[1];
  const double* dvi2 = g.dlv_inv[2];
  const long long c = c3(g, i, j, k);
  const long long s = AX == 0 ? 1 : AX == 1 ? sy : sz;
  double dTdx = 0., dTdy = 0., dTdz = 0., h = 0., f;
  // neighbours: cell c (right of the face) and c - s (left)
  if (AX == 0) dTdx = dvi0[i] * (T[c] - T[c - 1]);
  if (AX == 1) dTdy = dvi1[j] * (T[c] - T[c - sy]);
  if (AX == 2) dTdz = dvi2[k] * (T[c] - T[c - sz]);
  if (da.aniso) {
    double bxh, byh, bzh;
    if (AX == 0) {
      bxh = bf[c];
      byh = 0.5 * (w[BY * sv + c - 1] + w[BY * sv + c]);
      bzh = 0.5 * (w[BZ * sv + c - 1] + w[BZ * sv + c]);
    } else if (AX == 1) {
      byh = bf[sv + c];
      bxh = 0.5 * (w[BX * sv + c - sy] + w[BX * sv + c]);
      bzh = 0.5 * (w[BZ * sv + c - sy] + w[BZ * sv + c]);
    } else {
      bzh = bf[2 * sv + c];
      bxh = 0.5 * (w[BX * sv + c - sz] + w[BX * sv + c]);
      byh = 0.5 * (w[BY * sv + c - sz] + w[BY * sv + c]);
    }
#if BNZ_FAST_MATH
    // one reciprocal square root in place of a square root and a division
    double bhi = rsqrt(bxh * bxh + byh * byh + bzh * bzh + SMALL_NUM);
#else
    double bhi = 1. / sqrt(bxh * bxh + byh * byh + bzh * bzh + SMALL_NUM);
#endif
    double bxh1 = bxh * bhi, byh1 = byh * bhi, bzh1 = bzh * bhi;
    if (AX == 0) {
      h = fabs(bxh1);
      if (g.dims >= 2)  // tr_grad_lim_yx (syxv = 1 on Cartesian grids)
        dTdy = dlim(dlim((T[c - 1] - T[c - 1 - sy]) * dvi1[j], (T[c - 1 + sy] - T[c - 1]) * dvi1[j + 1]) * 1.,
                    dlim((T[c] - T[c - sy]) * dvi1[j], (T[c + sy] - T[c]) * dvi1[j + 1]) * 1.);
      if (g.dims >= 3)  // tr_grad_lim_zx
        dTdz = dlim(dlim((T[c - 1] - T[c - 1 - sz]) * dvi2[k], (T[c - 1 + sz] - T[c - 1]) * dvi2[k + 1]) * 1. * 1.,
                    dlim((T[c] - T[c - sz]) * dvi2[k], (T[c + sz] - T[c]) * dvi2[k + 1]) * 1. * 1.);
      f = -kappah * bxh1 * (bxh1 * dTdx + byh1 * dTdy + bzh1 * dTdz);
    } else if (AX == 1) {
      h = fabs(byh1);
      // tr_grad_lim_xy
      dTdx = dlim(dlim((T[c - sy] - T[c - sy - 1]) * dvi0[i], (T[c - sy + 1] - T[c - sy]) * dvi0[i + 1]),
                  dlim((T[c] - T[c - 1]) * dvi0[i], (T[c + 1] - T[c]) * dvi0[i + 1]));
      if (g.dims >= 3)  // tr_grad_lim_zy
        dTdz = dlim(dlim((T[c - sy] - T[c - sy - sz]) * dvi2[k], (T[c - sy + sz] - T[c - sy]) * dvi2[k + 1]) * 1. * 1.,
                    dlim((T[c] - T[c - sz]) * dvi2[k], (T[c + sz] - T[c]) * dvi2[k + 1]) * 1. * 1.);
      f = -kappah * byh1 * (bxh1 * dTdx + byh1 * dTdy + bzh1 * dTdz);
    } else {
      h = fabs(bzh1);
      // tr_grad_lim_xz, tr_grad_lim_yz
      dTdx = dlim(dlim((T[c - sz] - T[c - sz - 1]) * dvi0[i], (T[c - sz + 1] - T[c - sz]) * dvi0[i + 1]),
                  dlim((T[c] - T[c - 1]) * dvi0[i], (T[c + 1] - T[c]) * dvi0[i + 1]));
      dTdy = dlim(dlim((T[c - sz] - T[c - sz - sy]) * dvi1[j], (T[c - sz + sy] - T[c - sz]) * dvi1[j + 1]) * 1.,
                  dlim((T[c] - T[c - sy]) * dvi1[j], (T[c + sy] - T[c]) * dvi1[j + 1]) * 1.);
      f = -kappah * bzh1 * (bxh1 * dTdx + byh1 * dTdy + bzh1 * dTdz);
    }
  } else {
    if (AX == 0) {
      if (g.dims >= 2)  // tr_grad_yx
        dTdy = 0.25 * (((T[c - 1] - T[c - 1 - sy]) * dvi1[j] + (T[c - 1 + sy] - T[c - 1]) * dvi1[j + 1]) * 1. +
                       ((T[c] - T[c - sy]) * dvi1[j] + (T[c + sy] - T[c]) * dvi1[j + 1]) * 1.);
      if (g.dims >= 3)  // tr_grad_zx
        dTdz = 0.25 * (((T[c - sy] - T[c - sy - sz]) * dvi2[k] + (T[c - sy + sz] - T[c - sy]) * dvi2[k + 1]) * 1. * 1. +
                       ((T[c] - T[c - sz]) * dvi2[k] + (T[c + sz] - T[c]) * dvi2[k + 1]) * 1. * 1.);
      double dTds = sqrt(dTdx * dTdx + dTdy * dTdy + dTdz * dTdz + SMALL_NUM);
      h = fabs(dTdx / dTds);
      f = -kappah * dTdx;
    } else if (AX == 1) {
      dTdx = 0.25 * (((T[c - sy] - T[c - sy - 1]) * dvi0[i] + (T[c - sy + 1] - T[c - sy]) * dvi0[i + 1]) +
                     ((T[c] - T[c - 1]) * dvi0[i] + (T[c + 1] - T[c]) * dvi0[i + 1]));
      if (g.dims >= 3)  // tr_grad_zy
        dTdz = 0.25 * (((T[c - sy] - T[c - sy - sz]) * dvi2[k] + (T[c - sy + sz] - T[c - sy]) * dvi2[k + 1]) * 1. * 1. +
                       ((T[c] - T[c - sz]) * dvi2[k] + (T[c + sz] - T[c]) * dvi2[k + 1]) * 1. * 1.);
      double dTds = sqrt(dTdx * dTdx + dTdy * dTdy + dTdz * dTdz + SMALL_NUM);
      h = fabs(dTdy / dTds);
      f = -kappah * dTdy;
    } else {
      dTdx = 0.25 * (((T[c - sz] - T[c - sz - 1]) * dvi0[i] + (T[c - sz + 1] - T[c - sz]) * dvi0[i + 1]) +
                     ((T[c] - T[c - 1]) * dvi0[i] + (T[c + 1] - T[c]) * dvi0[i + 1]));
      dTdy = 0.25 * (((T[c - sz] - T[c - sz - sy]) * dvi1[j] + (T[c - sz + sy] - T[c - sz]) * dvi1[j + 1]) * 1. +
                     ((T[c] - T[c - sy]) * dvi1[j] + (T[c + sy] - T[c]) * dvi1[j + 1]) * 1.);
      double dTds = sqrt(dTdx * dTdx + dTdy * dTdy + dTdz * dTdz + SMALL_NUM);
      h = fabs(dTdz / dTds);
      f = -kappah * dTdz;
    }
  }
  if (da.sat) f = saturate(f, h, T[c - s], T[c], w[RHO * sv + c - s], w[RHO * sv + c]);
  return f;
}

// One whole RKL2 stage per cell (thcond_elec.pyx:75-94 with the operator of
// :118-338): the cell's six face fluxes from T (each interior face is formed
// by both of its cells with the same expression, so both see one value), the
// divergence M(p) = -(gamma-1) div q (thcond_elec.pyx:332-338) and the stage
// update p = mu p + nu p_(j-2) + (1 - mu - nu) p0 + dt (mut M(p) + gamt M(p0)).
// Only the cell's own p is read and written; the neighbours enter through T,
// which k_temp formed before the launch, so the face fluxes never see a
// pressure of this stage.  Stage 1 saves p0 and M(p0).  Per zone-stage this
// moves p, p_(j-2), p0, M(p0), the cell field and the face field, and T.
__global__ void k_stage(GridDev g, double* __restrict__ w, const double* __restrict__ bf,
                        const double* __restrict__ T, DiffArgs da, int3 lo, int3 hi, int first, double mu, double nu,
                        double mut, double gamt, const double* dtp) {
  const double dt = *dtp;
  const double gamm1 = g.gam - 1.;
  const int nxr = hi.x - lo.x + 1, nyr = hi.y - lo.y + 1, nzr = hi.z - lo.z + 1;
  const long long n = (long long)nxr * nyr * nzr;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = lo.x + (int)(t % nxr);
    const long long r = t / nxr;
    const int j = lo.y + (int)(r % nyr), k = lo.z + (int)(r / nyr);
    const long long c = c3(g, i, j, k);
    double v = -(face_flux<0>(g, w, bf, T, da, i + 1, j, k) - face_flux<0>(g, w, bf, T, da, i, j, k)) * gamm1 *
               g.dlf_inv[0][i];
    if (g.dims >= 2)
      v -= (face_flux<1>(g, w, bf, T, da, i, j + 1, k) - face_flux<1>(g, w, bf, T, da, i, j, k)) * gamm1 *
           g.dlf_inv[1][j];
    if (g.dims >= 3)
      v -= (face_flux<2>(g, w, bf, T, da, i, j, k + 1) - face_flux<2>(g, w, bf, T, da, i, j, k)) * gamm1 *
           g.dlf_inv[2][k];
    double* pp = w + PR * g.sv + c;
    if (first) {
      da.pres0[c] = *pp;
      da.dtemp0[c] = v;
    }
    const double a = *pp;
    *pp = (mu * a + nu * da.presm1[c] + (1. - mu - nu) * da.pres0[c] + dt * (mut * v + gamt * da.dtemp0[c]));
    da.presm1[c] = a;
  }
}

// thcond_elec.pyx:154-303, the field-aligned (anisotropic) face flux of
// face_flux<AX> with T and the limited transverse gradients read from a
// block's shared-memory tables: T over the tile and one cell around it
// (tT[(c * RY + b) * RX + a] is cell (x0 - 1 + a, y0 - 1 + b, z0 - 1 + c)),
// and for each direction d the inner limited gradient of every cell that a
// face's transverse gradient takes (util_diffusion.pyx:16-20), formed once
// per cell instead of once per face that uses it.  Same expressions, same
// bits as face_flux<AX>.
template <int TXC, int TYC, int TZC>
struct StageTab {
  static constexpr int RX = TXC + 2, RY = TYC + 2, RZ = TZC + 2;
  double T[RZ * RY * RX];
  double gx[RZ * RY * TXC];  // cells a = 1..TXC (the tile's x range), all b, c
  double gy[RZ * TYC * RX];  // cells b = 1..TYC, all a, c
  double gz[TZC * RY * RX];  // cells c = 1..TZC, all a, b
  __device__ int t(int a, int b, int c) const { return (c * RY + b) * RX + a; }
  __device__ int ix(int a, int b, int c) const { return (c * RY + b) * TXC + a - 1; }
  __device__ int iy(int a, int b, int c) const { return (c * TYC + b - 1) * RX + a; }
  __device__ int iz(int a, int b, int c) const { return ((c - 1) * RY + b) * RX + a; }
};

// the AX face whose right cell is (x0 - 1 + a, y0 - 1 + b, z0 - 1 + c) = (i, j, k)
template <int AX, int TXC, int TYC, int TZC>
__device__ __forceinline__ double face_flux_tab(const GridDev& g, const double* __restrict__ w,
                                                const double* __restrict__ bf, const StageTab<TXC, TYC, TZC>& S,
                                                const DiffArgs& da, int i, int j, int k, int a, int b, int cz) {
  const long long sy = g.nx, sz = (long long)g.nx * g.ny, sv = g.sv;
  const double k0 = da.kappa0;
  const double kappah = (2. * k0 * k0 / (k0 + k0 + SMALL_NUM));
  const long long c = c3(g, i, j, k);
  // the left cell's table coordinates
  const int al = AX == 0 ? a - 1 : a, bl = AX == 1 ? b - 1 : b, cl = AX == 2 ? cz - 1 : cz;
  double dTdx = 0., dTdy = 0., dTdz = 0., h, f;
  if (AX == 0) dTdx = g.dlv_inv[0][i] * (S.T[S.t(a, b, cz)] - S.T[S.t(al, bl, cl)]);
  if (AX == 1) dTdy = g.dlv_inv[1][j] * (S.T[S.t(a, b, cz)] - S.T[S.t(al, bl, cl)]);
  if (AX == 2) dTdz = g.dlv_inv[2][k] * (S.T[S.t(a, b, cz)] - S.T[S.t(al, bl, cl)]);
  double bxh, byh, bzh;
  if (AX == 0) {
    bxh = bf[c];
    byh = 0.5 * (w[BY * sv + c - 1] + w[BY * sv + c]);
    bzh = 0.5 * (w[BZ * sv + c - 1] + w[BZ * sv + c]);
  } else if (AX == 1) {
    byh = bf[sv + c];
    bxh = 0.5 * (w[BX * sv + c - sy] + w[BX * sv + c]);
    bzh = 0.5 * (w[BZ * sv + c - sy] + w[BZ * sv + c]);
  } else {
    bzh = bf[2 * sv + c];
    bxh = 0.5 * (w[BX * sv + c - sz] + w[BX * sv + c]);
    byh = 0.5 * (w[BY * sv + c - sz] + w[BY * sv + c]);
  }
#if BNZ_FAST_MATH
  double bhi = rsqrt(bxh * bxh + byh * byh + bzh * bzh + SMALL_NUM);
#else
  double bhi = 1. / sqrt(bxh * bxh + byh * byh + bzh * bzh + SMALL_NUM);
#endif
  double bxh1 = bxh * bhi, byh1 = byh * bhi, bzh1 = bzh * bhi;
  if (AX == 0) {
    h = fabs(bxh1);
    if (g.dims >= 2) dTdy = dlim(S.gy[S.iy(al, bl, cl)] * 1., S.gy[S.iy(a, b, cz)] * 1.);
    if (g.dims >= 3) dTdz = dlim(S.gz[S.iz(al, bl, cl)] * 1. * 1., S.gz[S.iz(a, b, cz)] * 1. * 1.);
    f = -kappah * bxh1 * (bxh1 * dTdx + byh1 * dTdy + bzh1 * dTdz);
  } else if (AX == 1) {
    h = fabs(byh1);
    dTdx = dlim(S.gx[S.ix(al, bl, cl)], S.gx[S.ix(a, b, cz)]);
    if (g.dims >= 3) dTdz = dlim(S.gz[S.iz(al, bl, cl)] * 1. * 1., S.gz[S.iz(a, b, cz)] * 1. * 1.);
    f = -kappah * byh1 * (bxh1 * dTdx + byh1 * dTdy + bzh1 * dTdz);
  } else {
    h = fabs(bzh1);
    dTdx = dlim(S.gx[S.ix(al, bl, cl)], S.gx[S.ix(a, b, cz)]);
    dTdy = dlim(S.gy[S.iy(al, bl, cl)] * 1., S.gy[S.iy(a, b, cz)] * 1.);
    f = -kappah * bzh1 * (bxh1 * dTdx + byh1 * dTdy + bzh1 * dTdz);
  }
  if (da.sat) f = saturate(f, h, S.T[S.t(al, bl, cl)], S.T[S.t(a, b, cz)], w[RHO * sv + c - (AX == 0 ? 1 : AX == 1 ? sy : sz)], w[RHO * sv + c]);
  return f;
}

// The same stage on a tile of TXC x TYC x TZC cells per block: the tile's
// face fluxes (each face once, the tile's far faces included) go to shared
// memory, then every cell forms M(p) from its six faces and updates.  Face
// values, divergence and update are the expressions of k_stage, so the two
// kernels give the same bits; the tile forms 1 + 1/T of a flux per face
// direction and cell instead of two.  With the field-aligned flux the block
// first stages T and each cell's limited transverse gradients (StageTab).
template <int TXC, int TYC, int TZC>
__global__ void __launch_bounds__(TXC * TYC * TZC) k_stage_tile(GridDev g, double* __restrict__ w,
                                                                 const double* __restrict__ bf,
                                                                 const double* __restrict__ T, DiffArgs da, int3 lo,
                                                                 int3 hi, int first, double mu, double nu, double mut,
                                                                 double gamt, const double* dtp) {
  constexpr int NX = (TXC + 1) * TYC * TZC, NY = TXC * (TYC + 1) * TZC, NZ = TXC * TYC * (TZC + 1);
  using Tab = StageTab<TXC, TYC, TZC>;
  __shared__ double sfx[NX], sfy[NY], sfz[NZ];
  __shared__ Tab S;
  const int nbx = (hi.x - lo.x + TXC) / TXC, nby = (hi.y - lo.y + TYC) / TYC;
  const int bx = blockIdx.x % nbx, by = (blockIdx.x / nbx) % nby, bz = blockIdx.x / (nbx * nby);
  const int x0 = lo.x + bx * TXC, y0 = lo.y + by * TYC, z0 = lo.z + bz * TZC;
  const int wx = min(TXC, hi.x - x0 + 1), wy = min(TYC, hi.y - y0 + 1), wz = min(TZC, hi.z - z0 + 1);
  if (da.aniso) {
    // T on the tile and one cell around it (the grid's cells only)
    for (int t = threadIdx.x; t < Tab::RX * Tab::RY * Tab::RZ; t += blockDim.x) {
      const int a = t % Tab::RX, r = t / Tab::RX, b = r % Tab::RY, cz = r / Tab::RY;
      const int x = x0 - 1 + a, y = y0 - 1 + b, z = z0 - 1 + cz;
      if (x < g.nx && y < g.ny && z < g.nz) S.T[t] = T[c3(g, x, y, z)];
    }
    __syncthreads();
    // each cell's inner limited gradient in each direction, where a face's
    // transverse gradient takes it: x gradients of the tile's x range, and so
    // on (the cell's own dvi, as face_flux<AX> forms them)
    constexpr int NGX = Tab::RZ * Tab::RY * TXC, NGY = Tab::RZ * TYC * Tab::RX, NGZ = TZC * Tab::RY * Tab::RX;
    for (int t = threadIdx.x; t < NGX + NGY + NGZ; t += blockDim.x) {
      if (t < NGX) {
        const int a = 1 + t % TXC, r = t / TXC, b = r % Tab::RY, cz = r / Tab::RY;
        const int x = x0 - 1 + a, y = y0 - 1 + b, z = z0 - 1 + cz;
        if (a > wx || y >= g.ny || z >= g.nz) continue;
        S.gx[t] = dlim((S.T[S.t(a, b, cz)] - S.T[S.t(a - 1, b, cz)]) * g.dlv_inv[0][x],
                       (S.T[S.t(a + 1, b, cz)] - S.T[S.t(a, b, cz)]) * g.dlv_inv[0][x + 1]);
      } else if (t < NGX + NGY) {
        if (g.dims < 2) continue;
        const int u = t - NGX;
        const int a = u % Tab::RX, r = u / Tab::RX, b = 1 + r % TYC, cz = r / TYC;
        const int x = x0 - 1 + a, y = y0 - 1 + b, z = z0 - 1 + cz;
        if (b > wy || x >= g.nx || z >= g.nz) continue;
        S.gy[u] = dlim((S.T[S.t(a, b, cz)] - S.T[S.t(a, b - 1, cz)]) * g.dlv_inv[1][y],
                       (S.T[S.t(a, b + 1, cz)] - S.T[S.t(a, b, cz)]) * g.dlv_inv[1][y + 1]);
      } else {
        if (g.dims < 3) continue;
        const int u = t - NGX - NGY;
        const int a = u % Tab::RX, r = u / Tab::RX, b = r % Tab::RY, cz = 1 + r / Tab::RY;
        const int x = x0 - 1 + a, y = y0 - 1 + b, z = z0 - 1 + cz;
        if (cz > wz || x >= g.nx || y >= g.ny) continue;
        S.gz[u] = dlim((S.T[S.t(a, b, cz)] - S.T[S.t(a, b, cz - 1)]) * g.dlv_inv[2][z],
                       (S.T[S.t(a, b, cz + 1)] - S.T[S.t(a, b, cz)]) * g.dlv_inv[2][z + 1]);
      }
    }
    __syncthreads();
  }
  // the faces of the full tile shape (compile-time index arithmetic); faces
  // past a partial tile's extent are skipped
  for (int t = threadIdx.x; t < NX + NY + NZ; t += blockDim.x) {
    if (t < NX) {
      const int fi = t % (TXC + 1), r = t / (TXC + 1), fj = r % TYC, fk = r / TYC;
      if (fi > wx || fj >= wy || fk >= wz) continue;
      sfx[t] = da.aniso ? face_flux_tab<0>(g, w, bf, S, da, x0 + fi, y0 + fj, z0 + fk, fi + 1, fj + 1, fk + 1)
                        : face_flux<0>(g, w, bf, T, da, x0 + fi, y0 + fj, z0 + fk);
    } else if (t < NX + NY) {
      if (g.dims < 2) continue;
      const int u = t - NX;
      const int fi = u % TXC, r = u / TXC, fj = r % (TYC + 1), fk = r / (TYC + 1);
      if (fi >= wx || fj > wy || fk >= wz) continue;
      sfy[u] = da.aniso ? face_flux_tab<1>(g, w, bf, S, da, x0 + fi, y0 + fj, z0 + fk, fi + 1, fj + 1, fk + 1)
                        : face_flux<1>(g, w, bf, T, da, x0 + fi, y0 + fj, z0 + fk);
    } else {
      if (g.dims < 3) continue;
      const int u = t - NX - NY;
      const int fi = u % TXC, r = u / TXC, fj = r % TYC, fk = r / TYC;
      if (fi >= wx || fj >= wy || fk > wz) continue;
      sfz[u] = da.aniso ? face_flux_tab<2>(g, w, bf, S, da, x0 + fi, y0 + fj, z0 + fk, fi + 1, fj + 1, fk + 1)
                        : face_flux<2>(g, w, bf, T, da, x0 + fi, y0 + fj, z0 + fk);
    }
  }
  __syncthreads();
  const int ci = threadIdx.x % TXC, cj = (threadIdx.x / TXC) % TYC, ck = threadIdx.x / (TXC * TYC);
  if (ci >= wx || cj >= wy || ck >= wz) return;
  const int i = x0 + ci, j = y0 + cj, k = z0 + ck;
  const double dt = *dtp;
  const double gamm1 = g.gam - 1.;
  const long long c = c3(g, i, j, k);
  double v = -(sfx[(ck * TYC + cj) * (TXC + 1) + ci + 1] - sfx[(ck * TYC + cj) * (TXC + 1) + ci]) * gamm1 *
             g.dlf_inv[0][i];
  if (g.dims >= 2)
    v -= (sfy[(ck * (TYC + 1) + cj + 1) * TXC + ci] - sfy[(ck * (TYC + 1) + cj) * TXC + ci]) * gamm1 *
         g.dlf_inv[1][j];
  if (g.dims >= 3)
    v -= (sfz[((ck + 1) * TYC + cj) * TXC + ci] - sfz[(ck * TYC + cj) * TXC + ci]) * gamm1 * g.dlf_inv[2][k];
  double* pp = w + PR * g.sv + c;
  if (first) {
    da.pres0[c] = *pp;
    da.dtemp0[c] = v;
  }
  const double a = *pp;
  *pp = (mu * a + nu * da.presm1[c] + (1. - mu - nu) * da.pres0[c] + dt * (mut * v + gamt * da.dtemp0[c]));
  da.presm1[c] = a;
}

// thcond_elec.pyx:355-466: max over active cells of kappa0 (gamma-1)/rho sum 1/dx^2
__global__ void k_diff_dt_max(GridDev g, const double* __restrict__ w, double kappa0, unsigned long long* slot) {
  double m = 0.;
  const double gamm1 = g.gam - 1.;
  const int nxa = g.i2 - g.i1 + 1, nya = g.j2 - g.j1 + 1, nza = g.k2 - g.k1 + 1;
  const long long n = (long long)nxa * nya * nza;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = g.i1 + (int)(t % nxa);
    long long r = t / nxa;
    int j = g.j1 + (int)(r % nya), k = g.k1 + (int)(r / nya);
    long long c = c3(g, i, j, k);
    double dsx = g.dlf[0][i], dsy = g.dlf[1][j], dsz = g.dlf[2][k];
    double ad = kappa0 / w[RHO * g.sv + c] * gamm1;
    double ad_dl2 = ad / sqr(dsx);
    if (g.dims >= 2) ad_dl2 = ad_dl2 + ad / sqr(dsy);
    if (g.dims >= 3) ad_dl2 = ad_dl2 + ad / sqr(dsz);
    if (ad_dl2 > m) m = ad_dl2;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (wid == 0) {
    m = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0 && m > 0.) atomicMax(slot, (unsigned long long)__double_as_longlong(m));
  }
}

}  // namespace diff
