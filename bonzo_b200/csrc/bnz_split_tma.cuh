// bnz_split_tma.cuh -- the split path's update kernel fed by TMA (3D grids
// whose Ntot_x is even, so that every row starts on a 16-byte boundary).
//
// k_update (bnz_split.cuh) reads about 45 values a cell straight from global
// memory and is bound by the latency of those loads.  Here a block marches a
// 32 x 8 column up z; per plane one thread issues six cp.async.bulk.tensor
// boxes (w^n, the x / y / z hydro fluxes, b^n and the edge EMFs, each box
// covering the column plus its upper faces, the z boxes two planes deep) into
// one of two shared-memory buffers, so that plane k+1 arrives while plane k
// computes.  Every wait is bounded.  The per-cell expressions are k_update's,
// so both kernels give the same bits.  Included inside the per-floating-point
// mode namespace, after bnz_fused.cuh and bnz_fused3d.cuh (their TMA helpers).
#pragma once

namespace split {

// TMA box width (even: covers the 32 cells and the upper face from an even
// column) and rows (the 8 rows and the upper face)
constexpr int TW = 34, TH = 9;
// box sizes in doubles, each sub-buffer padded to 128 bytes
constexpr int TB_W = 9 * TH * TW, TB_F = 6 * TH * TW, TB_FZ = 6 * 2 * TH * TW, TB_B = 3 * 2 * TH * TW;
constexpr int pad16(int n) { return (n + 15) & ~15; }
struct TmaBuf {
  // element (x, y, z, f) of a box of P planes at ((f * P + z) * TH + y) * TW + x
  double w[pad16(TB_W)];
  double fx[pad16(TB_F)];
  double fy[pad16(TB_F)];
  double fz[pad16(TB_FZ)];
  double b0[pad16(TB_B)];
  double ee[pad16(TB_B)];
};
constexpr unsigned TMA_TX_BYTES = 8u * (TB_W + 2 * TB_F + TB_FZ + 2 * TB_B);  // the boxes, whole
struct TmaSmem {
  TmaBuf buf[2];
  unsigned long long bar[2];
};
// the tensor maps a launch reads (128 bytes each): prim, the x / y / z
// fluxes, bfld, the b^n copy, the edge EMFs
enum { TM_PRIM = 0, TM_FX, TM_FY, TM_FZ, TM_BFLD, TM_BSAVE, TM_EE, TM_COUNT };

__device__ __forceinline__ void issue_plane(TmaBuf& B, unsigned long long* bar, const unsigned char* maps, int b0map,
                                            int x0, int y0, int k) {
  fused::tma::fence_async_shared();
  fused::tma::arrive_expect(bar, TMA_TX_BYTES);
  fused3::load_4d(B.w, bar, maps + TM_PRIM * 128, x0, y0, k, 0);
  fused3::load_4d(B.fx, bar, maps + TM_FX * 128, x0, y0, k, 0);
  fused3::load_4d(B.fy, bar, maps + TM_FY * 128, x0, y0, k, 0);
  fused3::load_4d(B.fz, bar, maps + TM_FZ * 128, x0, y0, k, 0);
  fused3::load_4d(B.b0, bar, maps + b0map * 128, x0, y0, k, 0);
  fused3::load_4d(B.ee, bar, maps + TM_EE * 128, x0, y0, k, 0);
}

// k_update of a 3D stage with its inputs staged by TMA (see the file
// comment); x0base is the update box's first column rounded down to even.
__global__ void __launch_bounds__(256, 1) k_update_tma(GridDev g, double* w1, const double* __restrict__ w0,
                                                       double* __restrict__ b1, double* __restrict__ bsave,
                                                       const unsigned char* __restrict__ maps, int b0map,
                                                       plain::Box box, int x0base, const double* dtp, double fac,
                                                       int src, double gx, double gy, double gz,
                                                       const double* __restrict__ fdriv, unsigned* err) {
  extern __shared__ __align__(128) unsigned char tma_smem[];
  TmaSmem& S = *reinterpret_cast<TmaSmem*>(tma_smem);
  const double dt = fac * *dtp;
  // a step of zero length leaves the state as it is (as k_update)
  if (dt == 0.) return;
  const long long sv = g.sv, sy = g.nx, sz = (long long)g.nx * g.ny;
  const double gv[3] = {gx, gy, gz};
  const bool grav = gx != 0. || gy != 0. || gz != 0.;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int x0 = x0base + (int)blockIdx.x * 32, y0 = box.lo.y + (int)blockIdx.y * 8;
  const int i = x0 + tx, j = y0 + ty;
  const bool live = i >= box.lo.x && i <= box.hi.x && j <= box.hi.y;
  const int kb = box.lo.z + (int)blockIdx.z * UPD_KZ, ke = min(kb + UPD_KZ - 1, box.hi.z);
  if (tid == 0) {
    fused::tma::bar_init(&S.bar[0], 1);
    fused::tma::bar_init(&S.bar[1], 1);
    fused::tma::fence_bar_init();
  }
  __syncthreads();
  if (tid == 0) issue_plane(S.buf[0], &S.bar[0], maps, b0map, x0, y0, kb);
  unsigned phase[2] = {0u, 0u};
  unsigned e = 0;
  double dsx = 0., dsy = 0., lvx = 0., lfx0 = 0., lfx1 = 0., dix = 0., lvy = 0., lfy0 = 0., lfy1 = 0., diy = 0.;
  if (live) {
    dsx = g.dlf[0][i];
    dsy = g.dlf[1][j];
    lvx = g.lv[0][i];
    lfx0 = g.lf[0][i];
    lfx1 = g.lf[0][i + 1];
    dix = g.dlf_inv[0][i];
    lvy = g.lv[1][j];
    lfy0 = g.lf[1][j];
    lfy1 = g.lf[1][j + 1];
    diy = g.dlf_inv[1][j];
  }
  for (int k = kb; k <= ke; ++k) {
    const int s = (k - kb) & 1;
    // the next plane into the other buffer, whose last reader passed the
    // barrier that ended the previous plane
    if (tid == 0 && k + 1 <= ke) issue_plane(S.buf[s ^ 1], &S.bar[s ^ 1], maps, b0map, x0, y0, k + 1);
    const bool ok = fused::tma::wait(&S.bar[s], phase[s]);
    phase[s] ^= 1u;
    if (__syncthreads_or(!ok)) {
      // a load that did not arrive: flag it, let the other buffer's load (if
      // any) land, and leave without writing
      if (tid == 0) {
        atomicOr(err, (unsigned)ERR_TIMEOUT);
        if (k + 1 <= ke) fused::tma::wait(&S.bar[s ^ 1], phase[s ^ 1]);
      }
      return;
    }
    if (live) {
      const TmaBuf& B = S.buf[s];
      const long long c = plain::cidx(g, i, j, k);
      auto FX = [&](int n, int dx) { return B.fx[(n * TH + ty) * TW + tx + dx]; };
      auto FY = [&](int n, int dy) { return B.fy[(n * TH + ty + dy) * TW + tx]; };
      auto FZ = [&](int n, int dz) { return B.fz[((n * 2 + dz) * TH + ty) * TW + tx]; };
      auto B0 = [&](int f, int dx, int dy, int dz) { return B.b0[((f * 2 + dz) * TH + ty + dy) * TW + tx + dx]; };
      auto EE = [&](int f, int dx, int dy, int dz) { return B.ee[((f * 2 + dz) * TH + ty + dy) * TW + tx + dx]; };
      // godunov.pyx:215-252
      const double dsz = g.dlf[2][k];
      const double vol = dsx * dsy * dsz;
      const double dtdv = dt / vol;
      const double dax = dsy * dsz;
      const double day = dsx * dsz;
      const double daz = dsx * dsy;
      double u[NM];
      {
        double wc[NM];
#pragma unroll
        for (int n = 0; n < NM; ++n) wc[n] = B.w[(n * TH + ty) * TW + tx];
        prim2cons(u, wc, g.gam);
      }
#pragma unroll
      for (int n = 0; n < BX; ++n) {
        double v = u[n] - dtdv * (dax * FX(n, 1) - dax * FX(n, 0));
        v -= dtdv * (day * FY(n, 1) - day * FY(n, 0));
        v -= dtdv * (daz * FZ(n, 1) - daz * FZ(n, 0));
        u[n] = v;
      }
      // ct.pyx:15-91 on the cell's faces (3D)
      auto bxf = [&](int dx) {
        const double dtda = dt / (dsy * dsz);
        double v = B0(0, dx, 0, 0);
        v -= dtda * (dsz * EE(2, dx, 1, 0) - dsz * EE(2, dx, 0, 0));
        v += dtda * (dsy * EE(1, dx, 0, 1) - dsy * EE(1, dx, 0, 0));
        return v;
      };
      auto byf = [&](int dy) {
        const double dtda = dt / (dsx * dsz);
        double v = B0(1, 0, dy, 0) + dtda * (dsz * EE(2, 1, dy, 0) - dsz * EE(2, 0, dy, 0));
        v -= dtda * (dsx * EE(0, 0, dy, 1) - dsx * EE(0, 0, dy, 0));
        return v;
      };
      auto bzf = [&](int dz) {
        const double dtda = dt / (dsx * dsy);
        double v = B0(2, 0, 0, dz) - dtda * (dsy * EE(1, 1, 0, dz) - dsy * EE(1, 0, 0, dz));
        v += dtda * (dsx * EE(0, 0, 1, dz) - dsx * EE(0, 0, 0, dz));
        return v;
      };
      const double bxl = bxf(0), byl = byf(0), bzl = bzf(0), bxr = bxf(1), byr = byf(1), bzr = bzf(1);
      b1[c] = bxl;
      b1[sv + c] = byl;
      b1[2 * sv + c] = bzl;
      const bool ux = i == box.hi.x, uy = j == box.hi.y, uz = k == box.hi.z;
      if (ux) b1[c + 1] = bxr;
      if (uy) b1[sv + c + sy] = byr;
      if (uz) b1[2 * sv + c + sz] = bzr;
      if (bsave) {
        bsave[c] = B0(0, 0, 0, 0);
        bsave[sv + c] = B0(1, 0, 0, 0);
        bsave[2 * sv + c] = B0(2, 0, 0, 0);
        if (ux) bsave[c + 1] = B0(0, 1, 0, 0);
        if (uy) bsave[sv + c + sy] = B0(1, 0, 1, 0);
        if (uz) bsave[2 * sv + c + sz] = B0(2, 0, 0, 1);
      }
      // ct.pyx:96-123
      u[BX] = ((lvx - lfx0) * bxl + (lfx1 - lvx) * bxr) * dix;
      u[BY] = ((lvy - lfy0) * byl + (lfy1 - lvy) * byr) * diy;
      u[BZ] = ((g.lv[2][k] - g.lf[2][k]) * bzl + (g.lf[2][k + 1] - g.lv[2][k]) * bzr) * g.dlf_inv[2][k];
      if (src) {
        // integrator.pyx:132-170 with the stage input w0
        double f[3];
        if (fdriv) {
          f[0] = fdriv[c];
          f[1] = fdriv[sv + c];
          f[2] = fdriv[2 * sv + c];
        }
        srcterm::apply(u, w0[c], w0[VX * sv + c], w0[VY * sv + c], w0[VZ * sv + c], gv, grav,
                       fdriv ? f : nullptr, dt);
      }
      // eos.pyx:13-44
      double ww[NM];
      cons2prim(ww, u, g.gam);
      e |= plain::check_prim(ww);
#pragma unroll
      for (int n = 0; n < NM; ++n) w1[n * sv + c] = ww[n];
    }
    __syncthreads();
  }
  if (e) atomicOr(err, e);
}

}  // namespace split
