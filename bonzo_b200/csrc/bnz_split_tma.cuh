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
// the tensor maps the split kernels read (128 bytes each): for the update,
// prim, the x / y / z fluxes, bfld, the b^n copy, the edge EMFs; for the PLM
// flux tiles, the predictor's prim (cons_s) in the boxes of the x, y, z sweeps
enum { TM_PRIM = 0, TM_FX, TM_FY, TM_FZ, TM_BFLD, TM_BSAVE, TM_EE, TM_WS0, TM_WS1, TM_WS2, TM_COUNT };

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

// Pencil tiles of the TMA-fed PLM flux kernel: one 4D box of all nine fields
// per tile (x sweep: 34 cells from an even column on 8 lines, 30 faces; y and
// z sweeps: 18 cells on 16 x-columns from an even column, 15 faces), staged
// with the fields in the global order (slot perm(n) holds local variable n).
template <int AX>
struct FTT {
  static constexpr int NA = AX == 0 ? 30 : 15;
  static constexpr int NB = AX == 0 ? 8 : 16;
  static constexpr int TAX = AX == 0 ? 1 : 0;
  static constexpr int OAX = AX == 2 ? 1 : 2;
  static constexpr int NS = AX == 0 ? 34 : 18;   // box extent along AX (row stride)
  static constexpr int NSU = NA + 3;             // staged cells used along AX
  static constexpr int DA = AX == 0 ? 1 : NB;
  static constexpr int WN = NB * NS;
  static constexpr unsigned BYTES = 8u * NM * WN;
  __device__ static constexpr int ws(int gf, int sa, int lb) {
    return AX == 0 ? (gf * NB + lb) * NS + sa : (gf * NS + sa) * NB + lb;
  }
  __device__ static constexpr int ds(int s, int la, int lb) {
    return AX == 0 ? (s * NB + lb) * (NA + 1) + la : (s * (NA + 1) + la) * NB + lb;
  }
  static_assert((NA + 1) * NB <= 256, "one slope cell per thread");
};

// dynamic shared memory of the flux kernel: two tile buffers (filled by TMA
// in turn), the slope table, two mbarriers
template <int AX>
struct FluxSmem {
  double w[2][NM * FTT<AX>::WN];
  double d[8 * FTT<AX>::NB * (FTT<AX>::NA + 1)];
  unsigned long long bar[2];
};

template <int LIM, class T, int AX>
__device__ __forceinline__ void cell_slopes_g(const double* p, double* sD, int la, int lb) {
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    if (n == BX) continue;
    const int q = plain::perm<AX>(n) * T::WN;
    sD[T::ds(slot8(n), la, lb)] = half_slope_split<LIM>(p[q - T::DA], p[q], p[q + T::DA]);
  }
}

// tile t of the flux box: its first face a0 along AX, first line b0 (even in
// x for the y and z sweeps) and plane o
template <int AX>
struct FluxTiles {
  int lo_a, hi_a, lo_b, hi_b, bb0, lo_o, na, nb, n;
  __device__ FluxTiles(const plain::Box& box) {
    using T = FTT<AX>;
    lo_a = ax_of(box.lo, AX);
    hi_a = ax_of(box.hi, AX);
    lo_b = ax_of(box.lo, T::TAX);
    hi_b = ax_of(box.hi, T::TAX);
    bb0 = AX == 0 ? lo_b : (lo_b & ~1);
    lo_o = ax_of(box.lo, T::OAX);
    na = (hi_a - lo_a + T::NA) / T::NA;
    nb = (hi_b - bb0 + T::NB) / T::NB;
    n = na * nb * (ax_of(box.hi, T::OAX) - lo_o + 1);
  }
  __device__ void at(int t, int& a0, int& b0, int& o) const {
    a0 = lo_a + (t % na) * FTT<AX>::NA;
    b0 = bb0 + ((t / na) % nb) * FTT<AX>::NB;
    o = lo_o + t / (na * nb);
  }
};

template <int AX>
__device__ __forceinline__ void issue_tile(double* dst, unsigned long long* bar, const unsigned char* maps, int a0,
                                           int b0, int o) {
  const void* map = maps + (TM_WS0 + AX) * 128;
  fused::tma::fence_async_shared();
  fused::tma::arrive_expect(bar, FTT<AX>::BYTES);
  if (AX == 0) fused3::load_4d(dst, bar, map, a0 - 2, b0, o, 0);
  else if (AX == 1) fused3::load_4d(dst, bar, map, b0, a0 - 2, o, 0);
  else fused3::load_4d(dst, bar, map, b0, o, a0 - 2, 0);
}

// k_flux_tile<AX, 1, RS> for the corrector of a 3D grid with even Ntot_x, as
// a persistent kernel: a block walks the tiles t = blockIdx.x + m gridDim.x,
// and while it computes one, the next one's cells arrive as a TMA box of the
// predictor's prim (map TM_WS0 + AX) into the other buffer.  Cells outside
// [vlo, vhi] are then overwritten from wfb (the step's prim), as k_flux_tile
// reads them.  The x sweep needs an even first face column minus two (lo_a
// even).  Same expressions, same bits.
template <int AX, int RS>
__global__ void __launch_bounds__(256, 2) k_flux_tile_tma(GridDev g, const unsigned char* __restrict__ maps,
                                                          const double* __restrict__ wfb, int3 vlo, int3 vhi,
                                                          const double* __restrict__ bf, double* __restrict__ F,
                                                          plain::Box box, int lim, int cp, unsigned* err) {
  using T = FTT<AX>;
  constexpr int NA = T::NA, NB = T::NB, NSU = T::NSU, DA = T::DA, WN = T::WN;
  extern __shared__ __align__(128) unsigned char flux_smem[];
  FluxSmem<AX>& S = *reinterpret_cast<FluxSmem<AX>*>(flux_smem);
  double* sD = S.d;
  const FluxTiles<AX> tl(box);
  const long long st[3] = {1, (long long)g.nx, (long long)g.nx * g.ny};
  const int N[3] = {g.nx, g.ny, g.nz};
  const long long sa = st[AX], sb = st[T::TAX], so = st[T::OAX];
  const int tid = threadIdx.x;
  const int la = AX == 0 ? tid % (NA + 1) : tid / NB;
  const int lb = AX == 0 ? tid / (NA + 1) : tid % NB;
  if ((int)blockIdx.x >= tl.n) return;
  if (tid == 0) {
    fused::tma::bar_init(&S.bar[0], 1);
    fused::tma::bar_init(&S.bar[1], 1);
    fused::tma::fence_bar_init();
  }
  __syncthreads();
  if (tid == 0) {
    int a0, b0, o;
    tl.at(blockIdx.x, a0, b0, o);
    issue_tile<AX>(S.w[0], &S.bar[0], maps, a0, b0, o);
  }
  unsigned phase[2] = {0u, 0u};
  unsigned e = 0;
  for (int t = blockIdx.x, m = 0; t < tl.n; t += gridDim.x, ++m) {
    const int s = m & 1;
    const bool more = t + (int)gridDim.x < tl.n;
    // the next tile into the other buffer, whose last reader passed the
    // barrier that ended the previous tile
    if (tid == 0 && more) {
      int a1, b1, o1;
      tl.at(t + gridDim.x, a1, b1, o1);
      issue_tile<AX>(S.w[s ^ 1], &S.bar[s ^ 1], maps, a1, b1, o1);
    }
    const bool ok = fused::tma::wait(&S.bar[s], phase[s]);
    phase[s] ^= 1u;
    if (__syncthreads_or(!ok)) {
      // a load that did not arrive: flag it, let the other buffer's load (if
      // any) land, and leave
      if (tid == 0) {
        atomicOr(err, (unsigned)ERR_TIMEOUT);
        if (more) fused::tma::wait(&S.bar[s ^ 1], phase[s ^ 1]);
      }
      return;
    }
    double* sW = S.w[s];
    int a0, b0, o;
    tl.at(t, a0, b0, o);
    // cells of the tile outside [vlo, vhi]: the step's prim
    const bool edge = a0 - 2 < ax_of(vlo, AX) || a0 - 2 + NSU - 1 > ax_of(vhi, AX) || b0 < ax_of(vlo, T::TAX) ||
                      b0 + NB - 1 > ax_of(vhi, T::TAX) || o < ax_of(vlo, T::OAX) || o > ax_of(vhi, T::OAX);
    if (edge) {
      for (int q = tid; q < NSU * NB; q += 256) {
        const int ia = AX == 0 ? q % NSU : q / NB;
        const int ib = AX == 0 ? q / NSU : q % NB;
        const int a = a0 - 2 + ia, b = b0 + ib;
        if (a < 0 || a >= N[AX] || b > tl.hi_b) continue;
        const bool in = a >= ax_of(vlo, AX) && a <= ax_of(vhi, AX) && b >= ax_of(vlo, T::TAX) &&
                        b <= ax_of(vhi, T::TAX) && o >= ax_of(vlo, T::OAX) && o <= ax_of(vhi, T::OAX);
        if (in) continue;
        const long long c = a * sa + b * sb + o * so;
#pragma unroll
        for (int gf = 0; gf < NM; ++gf) sW[T::ws(gf, ia, ib)] = wfb[gf * g.sv + c];
      }
      __syncthreads();
    }
    const bool line = lb < NB && b0 + lb >= tl.lo_b && b0 + lb <= tl.hi_b;
    {
      // the half slope of cell a0-1+la (staged index la+1), once per cell
      const int a = a0 - 1 + la;
      if (line && la <= NA && a >= 1 && a + 1 < N[AX] && a <= tl.hi_a) {
        const double* p = sW + T::ws(0, la + 1, lb);
        if (cp) {
          double wm[NM], wc[NM], wp[NM], d[NM];
#pragma unroll
          for (int n = 0; n < NM; ++n) {
            const int q = plain::perm<AX>(n) * WN;
            wm[n] = p[q - DA];
            wc[n] = p[q];
            wp[n] = p[q + DA];
          }
          plain::half_slopes_char_rt(lim, wm, wc, wp, g.gam, d);
#pragma unroll
          for (int n = 0; n < NM; ++n)
            if (n != BX) sD[T::ds(slot8(n), la, lb)] = d[n];
        } else if (lim == LIM_MC) {
          cell_slopes_g<LIM_MC, T, AX>(p, sD, la, lb);
        } else if (lim == LIM_MM) {
          cell_slopes_g<LIM_MM, T, AX>(p, sD, la, lb);
        } else {
          cell_slopes_g<LIM_VL, T, AX>(p, sD, la, lb);
        }
      }
    }
    __syncthreads();
    // the face a0+la between cells a0+la-1 and a0+la
    const int f = a0 + la, b = b0 + lb;
    if (line && la < NA && f <= tl.hi_a) {
      const long long c = f * sa + b * sb + o * so;
      const double* p = sW + T::ws(0, la + 2, lb);  // staged cell f
      double wL[NM], wR[NM];
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        if (n == BX) continue;
        const int q = plain::perm<AX>(n) * WN;
        wL[n] = p[q - DA] + sD[T::ds(slot8(n), la, lb)];
        wR[n] = p[q] - sD[T::ds(slot8(n), la + 1, lb)];
      }
      const double bx = bf[AX * g.sv + c];
      wL[BX] = bx;
      wR[BX] = bx;
      double fl[NM];
      riemann<RS, true>(fl, wL, wR, g.gam, e);
#pragma unroll
      for (int n = 0; n < NM; ++n)
        if (n != BX) F[plain::perm<AX>(n) * g.sv + c] = fl[n];
    }
    __syncthreads();
  }
  if (e) atomicOr(err, e);
}

}  // namespace split
