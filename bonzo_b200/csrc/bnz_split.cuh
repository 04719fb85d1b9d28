// bnz_split.cuh -- the split path: one launch per face direction, each face's
// flux formed once, then one fused update per stage.
//
// Where the plain path (bnz_plain.cuh) follows the reference loop by loop, the
// split path keeps its decomposition (fluxes and edge EMFs through HBM) and
// removes its costs:
//   * k_flux_tile: a block stages a pencil tile of cells (NB lines of NA faces
//     along the sweep axis, with the two-cell halo) in shared memory and forms
//     every cell's PLM half slopes once (reconstr_c.c:54-91), where
//     plain::k_flux forms both one-sided slopes of every face itself (the
//     donor-cell predictor, with no slopes to share, keeps plain::k_flux);
//   * k_ee forms the cell-centred EMF (ct.pyx:128-148) of the cells it needs
//     on the fly instead of reading a separate array;
//   * k_update: per cell, prim2cons of the step's input, the conservative
//     update (godunov.pyx:215-252), the face update (ct.pyx:15-91),
//     face-to-cell B (ct.pyx:96-123), the source terms
//     (integrator.pyx:132-170) and cons2prim (eos.pyx:13-44) in one pass,
//     where the plain path runs up to eight launches and keeps a conserved
//     state in HBM between them.
// A face is formed by exactly one block and no kernel waits on a barrier
// between Riemann solves (what bounds the z-marching chunk kernels).  Every
// expression is the plain path's, so the exact build is bitwise equal to it
// and to the oracle (the fast build's van Leer limiter differs: see
// half_slope_split).  The hydro build runs the same launches on zero fields.
// Included inside the per-floating-point-mode namespace, after bnz_plain.cuh
// and bnz_source.cuh.
#pragma once

namespace split {

using namespace dev;

// slope slot of variable n (the normal field has none)
__device__ __forceinline__ constexpr int slot8(int n) { return n < BX ? n : n - 1; }

// Pencil tiles of the flux kernel of axis AX: NA faces along AX on each of NB
// lines along the transverse axis TAX (y for the x sweep, x for the y and z
// sweeps, so that a warp's loads and stores run along x); OAX is the axis the
// block index walks one line at a time.  (NA + 1) NB = 256 threads: one slope
// cell per thread.  Shared arrays are laid out with x fastest, which keeps a
// warp's accesses on distinct banks.
template <int AX>
struct FT {
  static constexpr int NA = AX == 0 ? 31 : 15;
  static constexpr int NB = AX == 0 ? 8 : 16;
  static constexpr int TAX = AX == 0 ? 1 : 0;
  static constexpr int OAX = AX == 2 ? 1 : 2;
  static constexpr int NS = NA + 3;             // staged cells along AX
  static constexpr int NT = (NA + 1) * NB;
  static constexpr int DA = AX == 0 ? 1 : NB;   // stride along AX (staged cells and slopes)
  static constexpr int WN = NB * NS;            // stride between staged fields
  __device__ static constexpr int ws(int n, int sa, int lb) {  // staged cell sa of line lb
    return AX == 0 ? (n * NB + lb) * NS + sa : (n * NS + sa) * NB + lb;
  }
  __device__ static constexpr int ds(int s, int la, int lb) {  // slope of cell la of line lb
    return AX == 0 ? (s * NB + lb) * (NA + 1) + la : (s * (NA + 1) + la) * NB + lb;
  }
  static_assert(NT == 256, "one slope cell per thread");
};

__device__ __forceinline__ int ax_of(int3 v, int a) { return a == 0 ? v.x : a == 1 ? v.y : v.z; }

// reconstr_c.c:54-91 half slope; in the fast build the van Leer limiter's
// quotient 2ab/(a+b) is 2ab times the Newton-refined reciprocal of a + b
// (bnz_fastmath.cuh: within 2 ulp; ab > 0 makes a and b one-signed, so
// |a + b| >= 2 sqrt(ab) is a normal number)
template <int LIM>
__device__ __forceinline__ double half_slope_split(double wm, double wc, double wp) {
#if BNZ_FAST_MATH
  if (LIM == LIM_VL) {
    const double a = wc - wm, b = wp - wc, ab = a * b;
    return 0.5 * ((ab > 0.) ? (2. * ab) * bnz_nr_rcp(a + b) : 0.);
  }
#endif
  return half_slope<LIM>(wm, wc, wp);
}

// the eight half slopes (all but the normal field) of the staged cell at p
// into the slope table, one limiter for the whole loop
template <int LIM, class T>
__device__ __forceinline__ void cell_slopes(const double* p, double* sD, int la, int lb) {
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    if (n == BX) continue;
    sD[T::ds(slot8(n), la, lb)] = half_slope_split<LIM>(p[n * T::WN - T::DA], p[n * T::WN], p[n * T::WN + T::DA]);
  }
}

// Fluxes of the AX faces of `box` (face index along AX = the cell on its
// right), in the global variable order as plain::k_flux stores them (the
// normal field entry, which nothing reads, is not stored).  ORDER 0: donor
// cell (reconstr_c.c:8-22); ORDER 1: PLM with limiter lim (reconstr_c.c:29-91),
// in characteristic variables when cp.  Normal field from the face array.
// Cells outside [vlo, vhi] are read from wfb instead of w (the corrector reads
// the predictor's output, which covers cells 1..Ntot-2 of each active axis,
// and the step's input prim elsewhere).
template <int AX, int ORDER, int RS>
__global__ void __launch_bounds__(256, 2) k_flux_tile(GridDev g, const double* __restrict__ w,
                                                      const double* __restrict__ wfb, int3 vlo, int3 vhi,
                                                      const double* __restrict__ bf, double* __restrict__ F,
                                                      plain::Box box, int lim, int cp, unsigned* err) {
  using T = FT<AX>;
  constexpr int NA = T::NA, NB = T::NB, NS = T::NS, DA = T::DA, WN = T::WN;
  __shared__ double sW[NM * WN];
  __shared__ double sD[ORDER ? 8 * NB * (NA + 1) : 1];
  const int lo_a = ax_of(box.lo, AX), hi_a = ax_of(box.hi, AX);
  const int lo_b = ax_of(box.lo, T::TAX), hi_b = ax_of(box.hi, T::TAX);
  const int na = (hi_a - lo_a + NA) / NA, nb = (hi_b - lo_b + NB) / NB;
  const int ta = blockIdx.x % na, tb = (blockIdx.x / na) % nb, to = blockIdx.x / (na * nb);
  const int a0 = lo_a + ta * NA, b0 = lo_b + tb * NB, o = ax_of(box.lo, T::OAX) + to;
  const long long st[3] = {1, (long long)g.nx, (long long)g.nx * g.ny};
  const int N[3] = {g.nx, g.ny, g.nz};
  const long long sa = st[AX], sb = st[T::TAX], so = st[T::OAX];
  // stage cells a0-2 .. a0+NA of the NB lines, in the sweep frame's variable
  // order; cells outside the array are neither loaded nor used
  for (int t = threadIdx.x; t < NS * NB; t += T::NT) {
    const int ia = AX == 0 ? t % NS : t / NB;
    const int ib = AX == 0 ? t / NS : t % NB;
    const int a = a0 - 2 + ia, b = b0 + ib;
    if (a < 0 || a >= N[AX] || b > hi_b) continue;
    const long long c = a * sa + b * sb + o * so;
    const bool in = a >= ax_of(vlo, AX) && a <= ax_of(vhi, AX) && b >= ax_of(vlo, T::TAX) &&
                    b <= ax_of(vhi, T::TAX) && o >= ax_of(vlo, T::OAX) && o <= ax_of(vhi, T::OAX);
    const double* src = in ? w : wfb;
#pragma unroll
    for (int n = 0; n < NM; ++n) sW[T::ws(n, ia, ib)] = src[plain::perm<AX>(n) * g.sv + c];
  }
  __syncthreads();
  const int la = AX == 0 ? threadIdx.x % (NA + 1) : threadIdx.x / NB;
  const int lb = AX == 0 ? threadIdx.x / (NA + 1) : threadIdx.x % NB;
  if (ORDER == 1) {
    // the half slope of cell a0-1+la (staged index la+1), once per cell
    const int a = a0 - 1 + la;
    if (a >= 1 && a + 1 < N[AX] && a <= hi_a && b0 + lb <= hi_b) {
      const double* p = sW + T::ws(0, la + 1, lb);
      if (cp) {
        double wm[NM], wc[NM], wp[NM], d[NM];
#pragma unroll
        for (int n = 0; n < NM; ++n) {
          wm[n] = p[n * WN - DA];
          wc[n] = p[n * WN];
          wp[n] = p[n * WN + DA];
        }
        plain::half_slopes_char_rt(lim, wm, wc, wp, g.gam, d);
#pragma unroll
        for (int n = 0; n < NM; ++n)
          if (n != BX) sD[T::ds(slot8(n), la, lb)] = d[n];
      } else if (lim == LIM_MC) {
        cell_slopes<LIM_MC, T>(p, sD, la, lb);
      } else if (lim == LIM_MM) {
        cell_slopes<LIM_MM, T>(p, sD, la, lb);
      } else {
        cell_slopes<LIM_VL, T>(p, sD, la, lb);
      }
    }
    __syncthreads();
  }
  // the face a0+la between cells a0+la-1 and a0+la (threads la == NA have none)
  const int f = a0 + la, b = b0 + lb;
  if (la >= NA || f > hi_a || b > hi_b) return;
  const long long c = f * sa + b * sb + o * so;
  const double* p = sW + T::ws(0, la + 2, lb);  // staged cell f
  double wL[NM], wR[NM];
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    if (n == BX) continue;
    if (ORDER == 0) {
      wL[n] = p[n * WN - DA];
      wR[n] = p[n * WN];
    } else {
      wL[n] = p[n * WN - DA] + sD[T::ds(slot8(n), la, lb)];
      wR[n] = p[n * WN] - sD[T::ds(slot8(n), la + 1, lb)];
    }
  }
  const double bx = bf[AX * g.sv + c];
  wL[BX] = bx;
  wR[BX] = bx;
  unsigned e = 0;
  double fl[NM];
  riemann<RS, true>(fl, wL, wR, g.gam, e);
#pragma unroll
  for (int n = 0; n < NM; ++n)
    if (n != BX) F[plain::perm<AX>(n) * g.sv + c] = fl[n];
  if (e) atomicOr(err, e);
}

// k_ee and k_update: a thread walks UPD_KZ cells up z (blocks of 32 x 8
// columns) and asks L2 for the inputs of the cell two planes ahead while it
// computes, since a cell's loads outnumber what its registers hold in flight.
// (Staging each tile's inputs in shared memory by asynchronous copies first
// measured slower: 2.3 and 0.66 ms per 256^3 launch against 1.8 and 0.47.)
constexpr int UPD_KZ = 16;

__device__ __forceinline__ void prefetch_l2(const double* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// ct.pyx:128-148: component COMP of the cell-centred EMF -(v x B) of cell c
template <int COMP>
__device__ __forceinline__ double ec_at(const double* __restrict__ w, long long sv, long long c) {
  const double* q = w + c;
  if (COMP == 0) return -(q[VY * sv] * q[BZ * sv] - q[VZ * sv] * q[BY * sv]);
  if (COMP == 1) return (q[VX * sv] * q[BZ * sv] - q[VZ * sv] * q[BX * sv]);
  return -(q[VX * sv] * q[BY * sv] - q[VY * sv] * q[BX * sv]);
}

// ct.pyx:153-215 (interp_ee1): plain::k_ee with the cell EMFs formed from the
// stage input prim: w on [vlo, vhi], wfb elsewhere (as in k_flux_tile)
__global__ void k_ee(GridDev g, const double* __restrict__ w_in, const double* __restrict__ wfb, int3 vlo,
                     int3 vhi, const double* __restrict__ fx, const double* __restrict__ fy,
                     const double* __restrict__ fz, double* __restrict__ ee, plain::Box box) {
  const long long sv = g.sv, sy = g.nx, sz = (long long)g.nx * g.ny;
  const int i = box.lo.x + (int)(blockIdx.x * 32 + threadIdx.x);
  const int j = box.lo.y + (int)(blockIdx.y * 8 + threadIdx.y);
  if (i > box.hi.x || j > box.hi.y) return;
  const int kb = box.lo.z + (int)blockIdx.z * UPD_KZ, ke = min(kb + UPD_KZ - 1, box.hi.z);
  for (int k = kb; k <= ke; ++k) {
    const long long c = plain::cidx(g, i, j, k);
    if (k + 2 <= ke) {
      const long long p = c + 2 * sz;
#pragma unroll
      for (int n = VX; n <= BZ; ++n) {
        if (n == PR || n == PSC) continue;
        prefetch_l2(w_in + n * sv + p);
        prefetch_l2(w_in + n * sv + p - sy);
      }
      prefetch_l2(fx + BY * sv + p);
      prefetch_l2(fx + BY * sv + p - sy);
      prefetch_l2(fx + BZ * sv + p);
      prefetch_l2(fy + BX * sv + p);
      prefetch_l2(fy + BZ * sv + p);
      prefetch_l2(fz + BX * sv + p);
      prefetch_l2(fz + BY * sv + p);
      prefetch_l2(fz + BY * sv + p - sy);
    }
    // the source array of the cell (i - di, j - dj, k - dk)
    auto W = [&](int di, int dj, int dk) {
      const int x = i - di, y = j - dj, z = k - dk;
      return x >= vlo.x && x <= vhi.x && y >= vlo.y && y <= vhi.y && z >= vlo.z && z <= vhi.z ? w_in : wfb;
    };
    if (g.dims == 3) {
      ee[c] = (0.5 * (-fy[BZ * sv + c - sz] - fy[BZ * sv + c] + fz[BY * sv + c - sy] + fz[BY * sv + c]) -
               0.25 * (ec_at<0>(W(0, 1, 0), sv, c - sy) + ec_at<0>(W(0, 0, 0), sv, c) +
                       ec_at<0>(W(0, 1, 1), sv, c - sz - sy) + ec_at<0>(W(0, 0, 1), sv, c - sz)));
      ee[sv + c] = (0.5 * (-fz[BX * sv + c - 1] - fz[BX * sv + c] + fx[BZ * sv + c - sz] + fx[BZ * sv + c]) -
                    0.25 * (ec_at<1>(W(1, 0, 0), sv, c - 1) + ec_at<1>(W(0, 0, 0), sv, c) +
                            ec_at<1>(W(1, 0, 1), sv, c - sz - 1) + ec_at<1>(W(0, 0, 1), sv, c - sz)));
      ee[2 * sv + c] = (0.5 * (-fx[BY * sv + c - sy] - fx[BY * sv + c] + fy[BX * sv + c - 1] + fy[BX * sv + c]) -
                        0.25 * (ec_at<2>(W(1, 0, 0), sv, c - 1) + ec_at<2>(W(0, 0, 0), sv, c) +
                                ec_at<2>(W(1, 1, 0), sv, c - sy - 1) + ec_at<2>(W(0, 1, 0), sv, c - sy)));
    } else if (g.dims == 2) {
      ee[c] = -fy[BZ * sv + c];
      ee[sv + c] = fx[BZ * sv + c];
      ee[2 * sv + c] = (0.5 * (-fx[BY * sv + c - sy] - fx[BY * sv + c] + fy[BX * sv + c - 1] + fy[BX * sv + c]) -
                        0.25 * (ec_at<2>(W(1, 0, 0), sv, c - 1) + ec_at<2>(W(0, 0, 0), sv, c) +
                                ec_at<2>(W(1, 1, 0), sv, c - sy - 1) + ec_at<2>(W(0, 1, 0), sv, c - sy)));
    } else {
      ee[c] = -ec_at<0>(W(0, 0, 0), sv, c);
      ee[sv + c] = fx[BZ * sv + c];
      ee[2 * sv + c] = -fx[BY * sv + c];
    }
  }
}

// One stage's update of the cells of `box` (the stage's update range): the
// plain path's k_advance_hydro, k_advance_b (the cell's lower faces, and its
// upper ones on the range's last cells), k_interp_bc, k_source and
// k_cons2prim, with the same expressions.  The stage starts from U^n =
// prim2cons(wn) (what the plain path's cons array holds: eos.pyx:48-78 after
// the last step's boundary fill) and writes only the stage's prim w1 and
// faces b1; the conserved state of the step's end is formed from prim after
// the boundary fill, as the plain path does.  w0 is the stage input prim (the
// source terms).  w1 may be wn: a thread reads and writes only its own cell of
// them.  b0 must not be b1 (a cell reads its upper faces' old values, which
// the neighbour updates); bsave, when not null, receives the b0 faces the
// update reads (the step's b^n, for the corrector).
__global__ void __launch_bounds__(256, 2) k_update(GridDev g, double* w1, const double* wn,
                                                const double* __restrict__ w0, double* __restrict__ b1,
                                                const double* __restrict__ b0, double* __restrict__ bsave,
                                                const double* __restrict__ fx, const double* __restrict__ fy,
                                                const double* __restrict__ fz, const double* __restrict__ ee,
                                                plain::Box box, const double* dtp, double fac, int src,
                                                double gx, double gy, double gz, const double* __restrict__ fdriv,
                                                unsigned* err) {
  const double dt = fac * *dtp;
  // a step of zero length (an instance at its tmax) leaves the state as it
  // is, as the reference's loop does by not stepping
  if (dt == 0.) return;
  const long long sv = g.sv, sy = g.nx, sz = (long long)g.nx * g.ny;
  const double gv[3] = {gx, gy, gz};
  const bool grav = gx != 0. || gy != 0. || gz != 0.;
  unsigned e = 0;
  const int i = box.lo.x + (int)(blockIdx.x * 32 + threadIdx.x);
  const int j = box.lo.y + (int)(blockIdx.y * 8 + threadIdx.y);
  if (i > box.hi.x || j > box.hi.y) return;
  const int kb = box.lo.z + (int)blockIdx.z * UPD_KZ, ke = min(kb + UPD_KZ - 1, box.hi.z);
  const bool d2 = g.dims >= 2, d3 = g.dims >= 3;
  // the column's coordinates (loaded once: the stores below may alias them
  // for all the compiler knows)
  const double dsx = g.dlf[0][i], dsy = g.dlf[1][j];
  const double lvx = g.lv[0][i], lfx0 = g.lf[0][i], lfx1 = g.lf[0][i + 1], dix = g.dlf_inv[0][i];
  const double lvy = d2 ? g.lv[1][j] : 0., lfy0 = d2 ? g.lf[1][j] : 0., lfy1 = d2 ? g.lf[1][j + 1] : 0.;
  const double diy = d2 ? g.dlf_inv[1][j] : 0.;
  // carried up z: the cell's lower z-face values (fluxes, b0, the new face),
  // and the edge EMFs of its lower level
  double fzl[BX], bz0l = 0., bzl = 0.;
  double eyl[2], exl[2];  // ee_y at (i, i+1), ee_x at (j, j+1) on level k
  for (int k = kb; k <= ke; ++k) {
    const long long c = plain::cidx(g, i, j, k);
    const bool first = k == kb;
    if (k + 2 <= ke) {
      const long long p = c + 2 * sz;
#pragma unroll
      for (int n = 0; n < NM; ++n) prefetch_l2(wn + n * sv + p);
#pragma unroll
      for (int n = 0; n < BX; ++n) {
        prefetch_l2(fx + n * sv + p);
        prefetch_l2(fy + n * sv + p);
        prefetch_l2(fy + n * sv + p + sy);
        prefetch_l2(fz + n * sv + p);
      }
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        prefetch_l2(b0 + n * sv + p);
        prefetch_l2(ee + n * sv + p);
        prefetch_l2(ee + n * sv + p + sy);
      }
      if (src) {
#pragma unroll
        for (int n = 0; n <= VZ; ++n) prefetch_l2(w0 + n * sv + p);
      }
    }
    if (first) {
      if (d3) {
#pragma unroll
        for (int n = 0; n < BX; ++n) fzl[n] = fz[n * sv + c];
      }
      bz0l = b0[2 * sv + c];
      eyl[0] = ee[sv + c];
      eyl[1] = ee[sv + c + 1];
      exl[0] = d2 ? ee[c] : 0.;
      exl[1] = d2 ? ee[c + sy] : 0.;
    }
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
      for (int n = 0; n < NM; ++n) wc[n] = wn[n * sv + c];
      prim2cons(u, wc, g.gam);
    }
    double fzu[BX];
#pragma unroll
    for (int n = 0; n < BX; ++n) {
      const long long q = n * sv + c;
      double v = u[n] - dtdv * (dax * fx[q + 1] - dax * fx[q]);
      if (d2) v -= dtdv * (day * fy[q + sy] - day * fy[q]);
      if (d3) {
        fzu[n] = fz[q + sz];
        v -= dtdv * (daz * fzu[n] - daz * fzl[n]);
      }
      u[n] = v;
    }
    // ct.pyx:15-91 on the cell's faces; a face's expressions depend only on
    // its transverse indices, so the upper face is the lower one shifted
    // (the new lower z face is the cell below's upper one)
    double ez[2][2];  // ee_z at (i + dx, j + dy) on level k
    ez[0][0] = ee[2 * sv + c];
    ez[1][0] = ee[2 * sv + c + 1];
    ez[0][1] = d2 ? ee[2 * sv + c + sy] : 0.;
    ez[1][1] = d2 ? ee[2 * sv + c + sy + 1] : 0.;
    double eyu[2] = {0., 0.}, exu[2] = {0., 0.};  // level k + 1
    if (d3) {
      eyu[0] = ee[sv + c + sz];
      eyu[1] = ee[sv + c + sz + 1];
      exu[0] = ee[c + sz];
      exu[1] = ee[c + sz + sy];
    }
    const double bx0[2] = {b0[c], b0[c + 1]};
    const double by0[2] = {b0[sv + c], d2 ? b0[sv + c + sy] : 0.};
    const double bz0u = d3 ? b0[2 * sv + c + sz] : 0.;
    auto bxf = [&](int dx) {
      const double dtda = dt / (dsy * dsz);
      double v = bx0[dx];
      if (d2) v -= dtda * (dsz * ez[dx][1] - dsz * ez[dx][0]);
      if (d3) v += dtda * (dsy * eyu[dx] - dsy * eyl[dx]);
      return v;
    };
    auto byf = [&](int dy) {
      const double dtda = dt / (dsx * dsz);
      double v = by0[dy] + dtda * (dsz * ez[1][dy] - dsz * ez[0][dy]);
      if (d3) v -= dtda * (dsx * exu[dy] - dsx * exl[dy]);
      return v;
    };
    auto bzf = [&](double bz, const double* ey, const double* ex) {
      const double dtda = dt / (dsx * dsy);
      double v = bz - dtda * (dsy * ey[1] - dsy * ey[0]);
      if (d2) v += dtda * (dsx * ex[1] - dsx * ex[0]);
      return v;
    };
    if (first) bzl = bzf(bz0l, eyl, exl);
    const double bxl = bxf(0), byl = byf(0), bxr = bxf(1);
    const double byr = d2 ? byf(1) : 0.;
    const double bzr = d3 ? bzf(bz0u, eyu, exu) : 0.;
    b1[c] = bxl;
    b1[sv + c] = byl;
    b1[2 * sv + c] = bzl;
    const bool ux = i == box.hi.x, uy = d2 && j == box.hi.y, uz = d3 && k == box.hi.z;
    if (ux) b1[c + 1] = bxr;
    if (uy) b1[sv + c + sy] = byr;
    if (uz) b1[2 * sv + c + sz] = bzr;
    if (bsave) {
      bsave[c] = bx0[0];
      bsave[sv + c] = by0[0];
      bsave[2 * sv + c] = bz0l;
      if (ux) bsave[c + 1] = bx0[1];
      if (uy) bsave[sv + c + sy] = by0[1];
      if (uz) bsave[2 * sv + c + sz] = bz0u;
    }
    // ct.pyx:96-123
    u[BX] = ((lvx - lfx0) * bxl + (lfx1 - lvx) * bxr) * dix;
    if (d2)
      u[BY] = ((lvy - lfy0) * byl + (lfy1 - lvy) * byr) * diy;
    else
      u[BY] = byl;
    if (d3)
      u[BZ] = ((g.lv[2][k] - g.lf[2][k]) * bzl + (g.lf[2][k + 1] - g.lv[2][k]) * bzr) * g.dlf_inv[2][k];
    else
      u[BZ] = bzl;
    if (src) {
      // integrator.pyx:132-170 with the stage input w0
      double f[3];
      if (fdriv) {
        f[0] = fdriv[c];
        f[1] = fdriv[sv + c];
        f[2] = fdriv[2 * sv + c];
      }
      srcterm::apply(u, w0[c], w0[VX * sv + c], w0[VY * sv + c], w0[VZ * sv + c], gv, grav, fdriv ? f : nullptr,
                     dt);
    }
    // eos.pyx:13-44
    double ww[NM];
    cons2prim(ww, u, g.gam);
    e |= plain::check_prim(ww);
#pragma unroll
    for (int n = 0; n < NM; ++n) w1[n * sv + c] = ww[n];
    // the upper face values become the next cell's lower ones
    if (d3) {
#pragma unroll
      for (int n = 0; n < BX; ++n) fzl[n] = fzu[n];
    }
    bz0l = bz0u;
    bzl = bzr;
    eyl[0] = eyu[0];
    eyl[1] = eyu[1];
    exl[0] = exu[0];
    exl[1] = exu[1];
  }
  if (e) atomicOr(err, e);
}

}  // namespace split
