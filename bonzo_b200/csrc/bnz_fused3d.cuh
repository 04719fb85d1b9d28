// bnz_fused3d.cuh -- fused tile kernels of the 3D VL2 step: z-marching
// column chunks.
//
// One block takes a chunk of a 3D grid -- at most TX x TY cells in x and y,
// wz planes in z -- and marches up through its planes.  At plane q it forms,
// in shared memory, the x and y fluxes of plane q, the z fluxes of level q
// (the faces between planes q-1 and q), the cell-centred EMFs of plane q, the
// edge EMFs Ez of plane q and Ex, Ey of level q; then it updates plane q-1,
// whose fluxes and edge EMFs are complete.  Two slots of every per-plane
// array are kept (q-1 and q), so only the step's input and output state cross
// HBM: no interface state, flux or EMF is written out.
//   predictor (ORDER 0, vanleer.pyx:104-120): donor-cell states of w^n, the
//     ghost cells read through the boundary-condition index maps (ghosts are
//     never filled), the half-step update; writes ws and bs on cells
//     1..Ntot-2;
//   corrector (ORDER 1, vanleer.pyx:130-151): PLM half slopes of ws formed
//     once per cell and direction (x and y in the plane, z from three
//     planes), the full-step update of u^n = prim2cons(w^n) and b^n; writes
//     w^(n+1), b^(n+1) on the active cells and folds the next step's CFL
//     maximum into the instance's slot.
// The input planes are staged in a ring of shared-memory buffers, one or two
// planes ahead of use: the corrector's ws planes (chunk plus two cells of halo
// each side) by TMA (cp.async.bulk.tensor over a 4D map [field][z][y][x],
// completed on one mbarrier per buffer, every wait bounded), or by cp.async
// where the instance has no tensor map; the predictor's w^n / b^n planes
// (chunk plus one cell each side) by cp.async through the index maps, with
// the reflecting walls' sign flips and zero faces stored directly.
// Every expression keeps the plain path's order (bnz_plain.cuh: k_flux, k_ec,
// k_ee, k_advance_hydro, k_advance_b, k_interp_bc, cons2prim), so the exact
// build is bitwise equal to the plain path and the oracle.
// Included inside the per-floating-point-mode namespace, after bnz_fused.cuh.
#pragma once

namespace fused3 {

using namespace dev;
using Inst = FusedInst3;
using Tile = FusedTile3;
using fused::AxisMap;
using fused::FastDiv;
using fused::map_cell;
using fused::map_face;

constexpr int TX = F3_TX, TY = F3_TY;  // cells of a chunk in x and y (at most)
constexpr int NT = 512;         // threads per block
constexpr int NF = 8;           // stored flux values: 6 hydro + the 2 field fluxes the EMFs need
constexpr int RX = TX + 2, RY = TY + 2, RC = RX * RY;  // the chunk plus one ring of cells
constexpr int NFX = (TX + 1) * RY;                       // x faces x0..x0+wx on rows y0-1..y0+wy
constexpr int NFY = RX * (TY + 1);                       // y faces y0..y0+wy on columns x0-1..x0+wx
constexpr int NEZ = (TX + 1) * (TY + 1);                 // Ez corners of a plane
constexpr int NEX = TX * (TY + 1);                       // Ex edges of a level
constexpr int NEY = (TX + 1) * TY;                       // Ey edges of a level
// the corrector's ws box: the chunk plus two cells each side, from an even
// column (16-byte rule for FP64 TMA); TX + 5 columns at most
constexpr int BW = F3_BW, BH = F3_BH, BC = BW * BH;
constexpr int WB1 = (NM * BC + 15) / 16 * 16;        // doubles per corrector buffer (128-byte multiple)
constexpr int WB0 = ((NM + 3) * RC + 15) / 16 * 16;  // predictor buffer: 9 prim + 3 faces on the ring region
constexpr unsigned BOX_BYTES = NM * BC * sizeof(double);

template <int ORDER>
struct Lay {
  static constexpr int NWB = 4;  // ring depth
  static constexpr int WB = ORDER ? WB1 : WB0;
  static constexpr int oW = 0;
  static constexpr int oSX = oW + NWB * WB;               // corrector: x slopes of the plane
  static constexpr int oSY = oSX + (ORDER ? 8 * RC : 0);  // y slopes
  static constexpr int oDZ = oSY + (ORDER ? 8 * RC : 0);  // z slopes, two planes
  static constexpr int oFX = oDZ + (ORDER ? 16 * RC : 0);
  static constexpr int oFY = oFX + 2 * NF * NFX;
  static constexpr int oFZ = oFY + 2 * NF * NFY;
  static constexpr int oEC = oFZ + 2 * NF * RC;
  static constexpr int oEZ = oEC + 2 * 3 * RC;
  static constexpr int oEX = oEZ + 2 * NEZ;
  static constexpr int oEY = oEX + 2 * NEX;
  static constexpr int total = oEY + 2 * NEY;
  static constexpr size_t bytes = 128 + sizeof(double) * (size_t)total;
};
static_assert(Lay<1>::bytes <= 227 * 1024 && Lay<0>::bytes <= 227 * 1024, "one block per SM");
static_assert(WB1 * sizeof(double) % 128 == 0 && BOX_BYTES <= WB1 * sizeof(double), "TMA buffers");

// Index maps of a chunk (array coordinates; max-size strides).
struct Geo {
  int x0, y0, wx, wy;
  int xs, ys;  // corrector box origin
  __device__ __forceinline__ int ri(int i, int j) const { return (j - y0 + 1) * RX + (i - x0 + 1); }
  __device__ __forceinline__ int fxi(int i, int j) const { return (j - y0 + 1) * (TX + 1) + (i - x0); }
  __device__ __forceinline__ int fyi(int i, int j) const { return (j - y0) * RX + (i - x0 + 1); }
  __device__ __forceinline__ int ezi(int i, int j) const { return (j - y0) * (TX + 1) + (i - x0); }
  __device__ __forceinline__ int exi(int i, int j) const { return (j - y0) * TX + (i - x0); }
  __device__ __forceinline__ int eyi(int i, int j) const { return (j - y0) * (TX + 1) + (i - x0); }
  __device__ __forceinline__ int wi1(int i, int j) const { return (j - ys) * BW + (i - xs); }
};

// A staged plane: field n at cell (i, j).
template <int ORDER>
struct Plane {
  const double* p;
  __device__ __forceinline__ double operator()(const Geo& G, int n, int i, int j) const {
    return ORDER ? p[n * BC + G.wi1(i, j)] : p[n * RC + G.ri(i, j)];
  }
};

__device__ __forceinline__ AxisMap axis_map3(const Inst& I, int ax) {
  AxisMap m;
  m.a1 = I.ng;
  m.a2 = I.ng + I.N[ax] - 1;
  m.n = I.N[ax];
  m.f0 = I.bc[ax][0];
  m.f1 = I.bc[ax][1];
  m.face_aware = I.face_aware;
  return m;
}

// face component COMP at (i, j, k) with ghost indices mapped (the 3D form of
// fused::load_face: the normal axis through the face map, the tangential
// axes through the cell map without sign flips)
template <int COMP>
__device__ __forceinline__ double face_mapped(const Inst& I, const double* __restrict__ b, int i, int j, int k,
                                              const AxisMap& mx, const AxisMap& my, const AxisMap& mz) {
  bool f = false, z = false, t;
  const int si = COMP == 0 ? map_face(i, mx, f, z) : map_cell(i, mx, t);
  const int sj = COMP == 1 ? map_face(j, my, f, z) : map_cell(j, my, t);
  const int sk = COMP == 2 ? map_face(k, mz, f, z) : map_cell(k, mz, t);
  if (z) return 0.;
  const double v = b[COMP * I.sv + ((long long)sk * I.ny + sj) * I.nx + si];
  return f ? -v : v;
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(fused::tma::saddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void load_4d(void* dst, unsigned long long* bar, const void* map, int x, int y, int z,
                                        int f) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(fused::tma::saddr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(f), "r"(fused::tma::saddr(bar))
      : "memory");
}

// The predictor's plane p (w^n: 9 fields, b^n: 3 faces) on the ring region
// (cells x0-1..x0+wx, y0-1..y0+wy) through the index maps, by cp.async;
// mirrored values (sign flips) and zero faces of reflecting walls are stored
// directly.
__device__ __forceinline__ void stage_pred_plane(const Inst& I, const Geo& G, int p, const double* __restrict__ w,
                                                 const double* __restrict__ b, double* dst) {
  const AxisMap mx = axis_map3(I, 0), my = axis_map3(I, 1), mz = axis_map3(I, 2);
  const int rw = G.wx + 2, nc = rw * (G.wy + 2);
  FastDiv dn, dr;
  dn.set(nc);
  dr.set(rw);
  bool fzp;
  const int skc = map_cell(p, mz, fzp);
  for (int t = threadIdx.x; t < (NM + 3) * nc; t += NT) {
    const int f = dn.div(t), u = t - f * nc;
    const int cj = dr.div(u), ci = u - cj * rw;
    const int i = G.x0 - 1 + ci, j = G.y0 - 1 + cj;
    double* d = dst + f * RC + G.ri(i, j);
    const double* src;
    bool flip = false, zero = false;
    if (f < NM) {
      bool fx, fy;
      const int si = map_cell(i, mx, fx), sj = map_cell(j, my, fy);
      flip = (fx && (f == VX || f == BX)) || (fy && (f == VY || f == BY)) || (fzp && (f == VZ || f == BZ));
      src = w + f * I.sv + ((long long)skc * I.ny + sj) * I.nx + si;
    } else {
      const int comp = f - NM;
      bool t0, t1;
      int si, sj, sk;
      if (comp == 0) {
        si = map_face(i, mx, flip, zero);
        sj = map_cell(j, my, t1);
        sk = skc;
      } else if (comp == 1) {
        si = map_cell(i, mx, t0);
        sj = map_face(j, my, flip, zero);
        sk = skc;
      } else {
        si = map_cell(i, mx, t0);
        sj = map_cell(j, my, t1);
        sk = map_face(p, mz, flip, zero);
      }
      src = b + comp * I.sv + ((long long)sk * I.ny + sj) * I.nx + si;
    }
    if (zero) *d = 0.;
    else if (flip) *d = -*src;
    else cp_async8(d, src);
  }
}

// The corrector's ws plane p on the TMA box layout by cp.async (instances
// without a tensor map): cells x0-2..x0+wx+1, y0-2..y0+wy+1.
__device__ __forceinline__ void stage_ws_plane(const Inst& I, const Geo& G, int p, double* dst) {
  const int rw = G.wx + 4, nc = rw * (G.wy + 4);
  FastDiv dn, dr;
  dn.set(nc);
  dr.set(rw);
  for (int t = threadIdx.x; t < NM * nc; t += NT) {
    const int f = dn.div(t), u = t - f * nc;
    const int cj = dr.div(u), ci = u - cj * rw;
    const int i = G.x0 - 2 + ci, j = G.y0 - 2 + cj;
    cp_async8(dst + f * BC + G.wi1(i, j), I.ws + f * I.sv + ((long long)p * I.ny + j) * I.nx + i);
  }
}

// The corrector's half slopes of plane q along AX (x, y in the plane; z from
// planes q-1, q, q+1) at cell (i, j), into D (8 fields of RC): the values
// reconstr_linear forms per face (reconstr_c.c:54-91), once per cell.
template <int AX, int LIM>
__device__ __forceinline__ void slope_cell(const Geo& G, const Plane<1>& Wm, const Plane<1>& Wc, const Plane<1>& Wp,
                                           int i, int j, int cp, double gam, double* D) {
  const int r = G.ri(i, j);
  const int im = AX == 0 ? i - 1 : i, ip = AX == 0 ? i + 1 : i;
  const int jm = AX == 1 ? j - 1 : j, jp = AX == 1 ? j + 1 : j;
  const Plane<1>& A = AX == 2 ? Wm : Wc;
  const Plane<1>& C = AX == 2 ? Wp : Wc;
  if (cp) {
    double wm[NM], wc[NM], wp[NM], d[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      const int gv = plain::perm<AX>(n);
      wm[n] = A(G, gv, im, jm);
      wc[n] = Wc(G, gv, i, j);
      wp[n] = C(G, gv, ip, jp);
    }
    half_slopes_char<LIM>(wm, wc, wp, gam, d);
#pragma unroll
    for (int n = 0; n < NM; ++n)
      if (n != BX) D[fused::slot8(n) * RC + r] = d[n];
  } else {
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      if (n == BX) continue;
      const int gv = plain::perm<AX>(n);
      D[fused::slot8(n) * RC + r] = half_slope<LIM>(A(G, gv, im, jm), Wc(G, gv, i, j), C(G, gv, ip, jp));
    }
  }
}

template <int ORDER>
struct Smem3 {
  double* W;  // ring base
  double *SX, *SY, *DZ, *FX, *FY, *FZ, *EC, *EZ, *EX, *EY;
  __device__ __forceinline__ void set(double* s) {
    using L = Lay<ORDER>;
    W = s + L::oW;
    SX = s + L::oSX;
    SY = s + L::oSY;
    DZ = s + L::oDZ;
    FX = s + L::oFX;
    FY = s + L::oFY;
    FZ = s + L::oFZ;
    EC = s + L::oEC;
    EZ = s + L::oEZ;
    EX = s + L::oEX;
    EY = s + L::oEY;
  }
  // the two slots of the per-plane arrays: plane (or level) q in slot q & 1
  __device__ __forceinline__ double* fx(int q) const { return FX + (q & 1) * NF * NFX; }
  __device__ __forceinline__ double* fy(int q) const { return FY + (q & 1) * NF * NFY; }
  __device__ __forceinline__ double* fz(int q) const { return FZ + (q & 1) * NF * RC; }
  __device__ __forceinline__ double* ec(int q) const { return EC + (q & 1) * 3 * RC; }
  __device__ __forceinline__ double* ez(int q) const { return EZ + (q & 1) * NEZ; }
  __device__ __forceinline__ double* ex(int q) const { return EX + (q & 1) * NEX; }
  __device__ __forceinline__ double* ey(int q) const { return EY + (q & 1) * NEY; }
  __device__ __forceinline__ double* dz(int q) const { return DZ + (q & 1) * 8 * RC; }
};

// Everything one chunk's phases read and write.
template <int ORDER>
struct March {
  const Inst* I;
  Geo G;
  Smem3<ORDER> S;
  int parity, cp, pbase;
  double dt;
  AxisMap mx, my, mz;
  int i2, j2, k2, ilast, jlast, klast;
  long long sy, sz;
  __device__ __forceinline__ double* buf(int p) const { return S.W + ((p - pbase) & 3) * Lay<ORDER>::WB; }
  // the z faces and z slopes of the ring region skip its four corners (no
  // edge EMF or cell update reads them)
  __device__ __forceinline__ bool corner(int ci, int cj) const {
    return (ci == 0 || ci == G.wx + 1) && (cj == 0 || cj == G.wy + 1);
  }
};

// Pre-flux items of plane q (ORDER 1: x slopes with E_c, y slopes, z slopes;
// ORDER 0: E_c only); u < npre(M).
template <int ORDER>
__device__ __forceinline__ int npre(const March<ORDER>& M) {
  const int nc = (M.G.wx + 2) * (M.G.wy + 2);
  return ORDER ? 3 * nc : nc;
}

template <int ORDER, int LIM>
__device__ __forceinline__ void pre_item(const March<ORDER>& M, int q, int u) {
  const Geo& G = M.G;
  const int rw = G.wx + 2, nc = rw * (G.wy + 2);
  const int dir = ORDER ? (u >= 2 * nc ? 2 : (u >= nc ? 1 : 0)) : 0;
  const int v = u - dir * nc;
  const int cj = v / rw, ci = v - cj * rw;
  const int i = G.x0 - 1 + ci, j = G.y0 - 1 + cj;
  const Plane<ORDER> Wq{M.buf(q)};
  if (dir == 0) {
    // cell-centred E (ct.pyx:128-148) of plane q
    const int r = G.ri(i, j);
    double* EC = M.S.ec(q);
    const double vx = Wq(G, VX, i, j), vy = Wq(G, VY, i, j), vz = Wq(G, VZ, i, j);
    const double bx = Wq(G, BX, i, j), by = Wq(G, BY, i, j), bz = Wq(G, BZ, i, j);
    EC[r] = -(vy * bz - vz * by);
    EC[RC + r] = (vx * bz - vz * bx);
    EC[2 * RC + r] = -(vx * by - vy * bx);
  }
  if constexpr (ORDER == 1) {
    const Plane<1> Wm{M.buf(q - 1)}, Wc{M.buf(q)}, Wp{M.buf(q + 1)};
    if (dir == 0) slope_cell<0, LIM>(G, Wm, Wc, Wp, i, j, M.cp, M.I->gam, M.S.SX);
    else if (dir == 1) slope_cell<1, LIM>(G, Wm, Wc, Wp, i, j, M.cp, M.I->gam, M.S.SY);
    else if (!M.corner(ci, cj)) slope_cell<2, LIM>(G, Wm, Wc, Wp, i, j, M.cp, M.I->gam, M.S.dz(q));
  }
}

// Flux item t of plane q: x faces, y faces, then (unless first) the z faces
// of level q, one Riemann call site for the three directions.
template <int ORDER, int RS>
__device__ __forceinline__ void flux_item(const March<ORDER>& M, int q, int t, int nfx, int nfy, unsigned& e) {
  const Geo& G = M.G;
  const Inst& I = *M.I;
  const int rw = G.wx + 2;
  const int dir = t >= nfx + nfy ? 2 : (t >= nfx ? 1 : 0);
  int i, j;
  if (dir == 0) {
    const int fj = t / (G.wx + 1), fi = t - fj * (G.wx + 1);
    i = G.x0 + fi;
    j = G.y0 - 1 + fj;
  } else if (dir == 1) {
    const int u = t - nfx;
    const int fj = u / rw, fi = u - fj * rw;
    i = G.x0 - 1 + fi;
    j = G.y0 + fj;
  } else {
    const int u = t - nfx - nfy;
    const int cj = u / rw, ci = u - cj * rw;
    if (M.corner(ci, cj)) return;
    i = G.x0 - 1 + ci;
    j = G.y0 - 1 + cj;
  }
  const Plane<ORDER> Wq{M.buf(q)};
  double wL[NM], wR[NM];
  double bn;
  if (dir == 0) {
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      if (n == BX) continue;
      if (ORDER == 1) {
        wL[n] = Wq(G, n, i - 1, j) + M.S.SX[fused::slot8(n) * RC + G.ri(i - 1, j)];
        wR[n] = Wq(G, n, i, j) - M.S.SX[fused::slot8(n) * RC + G.ri(i, j)];
      } else {
        wL[n] = Wq(G, n, i - 1, j);
        wR[n] = Wq(G, n, i, j);
      }
    }
    bn = ORDER ? I.bs[q * M.sz + j * M.sy + i] : Wq(G, NM, i, j);
  } else if (dir == 1) {
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      if (n == BX) continue;
      const int gv = plain::perm<1>(n);
      if (ORDER == 1) {
        wL[n] = Wq(G, gv, i, j - 1) + M.S.SY[fused::slot8(n) * RC + G.ri(i, j - 1)];
        wR[n] = Wq(G, gv, i, j) - M.S.SY[fused::slot8(n) * RC + G.ri(i, j)];
      } else {
        wL[n] = Wq(G, gv, i, j - 1);
        wR[n] = Wq(G, gv, i, j);
      }
    }
    bn = ORDER ? I.bs[I.sv + q * M.sz + j * M.sy + i] : Wq(G, NM + 1, i, j);
  } else {
    const Plane<ORDER> Wm{M.buf(q - 1)};
    const double* DZm = M.S.dz(q - 1);
    const double* DZc = M.S.dz(q);
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      if (n == BX) continue;
      const int gv = plain::perm<2>(n);
      if (ORDER == 1) {
        wL[n] = Wm(G, gv, i, j) + DZm[fused::slot8(n) * RC + G.ri(i, j)];
        wR[n] = Wq(G, gv, i, j) - DZc[fused::slot8(n) * RC + G.ri(i, j)];
      } else {
        wL[n] = Wm(G, gv, i, j);
        wR[n] = Wq(G, gv, i, j);
      }
    }
    bn = ORDER ? I.bs[2 * I.sv + q * M.sz + j * M.sy + i] : Wq(G, NM + 2, i, j);
  }
  wL[BX] = wR[BX] = bn;
  double f[NM];
  riemann<RS, true>(f, wL, wR, I.gam, e);
  // local sweep frame -> global variables (godunov.pyx:297-324)
  if (dir == 0) {
    double* FX = M.S.fx(q);
    const int o = G.fxi(i, j);
#pragma unroll
    for (int n = 0; n < 6; ++n) FX[n * NFX + o] = f[n];
    FX[6 * NFX + o] = f[BY];  // fx[BY]
    FX[7 * NFX + o] = f[BZ];  // fx[BZ]
  } else if (dir == 1) {
    double* FY = M.S.fy(q);
    const int o = G.fyi(i, j);
    FY[0 * NFY + o] = f[RHO];
    FY[1 * NFY + o] = f[VZ];  // global MX
    FY[2 * NFY + o] = f[VX];  // global MY
    FY[3 * NFY + o] = f[VY];  // global MZ
    FY[4 * NFY + o] = f[EN];
    FY[5 * NFY + o] = f[PSC];
    FY[6 * NFY + o] = f[BZ];  // fy[BX]
    FY[7 * NFY + o] = f[BY];  // fy[BZ]
  } else {
    double* FZ = M.S.fz(q);
    const int o = G.ri(i, j);
    FZ[0 * RC + o] = f[RHO];
    FZ[1 * RC + o] = f[VY];  // global MX
    FZ[2 * RC + o] = f[VZ];  // global MY
    FZ[3 * RC + o] = f[VX];  // global MZ
    FZ[4 * RC + o] = f[EN];
    FZ[5 * RC + o] = f[PSC];
    FZ[6 * RC + o] = f[BY];  // fz[BX]
    FZ[7 * RC + o] = f[BZ];  // fz[BY]
  }
}

// Edge item t (ct.pyx:153-215, interp_ee1): Ez corners of plane q, then
// (unless first) Ex and Ey edges of level q.
template <int ORDER>
__device__ __forceinline__ void edge_item(const March<ORDER>& M, int q, int t, int nez, int nex) {
  const Geo& G = M.G;
  const double *FXc = M.S.fx(q), *FYc = M.S.fy(q), *FZc = M.S.fz(q), *ECc = M.S.ec(q);
  if (t < nez) {
    const int cj = t / (G.wx + 1), ci = t - cj * (G.wx + 1);
    const int i = G.x0 + ci, j = G.y0 + cj;
    M.S.ez(q)[G.ezi(i, j)] =
        (0.5 * (-FXc[6 * NFX + G.fxi(i, j - 1)] - FXc[6 * NFX + G.fxi(i, j)] + FYc[6 * NFY + G.fyi(i - 1, j)] +
                FYc[6 * NFY + G.fyi(i, j)]) -
         0.25 * (ECc[2 * RC + G.ri(i - 1, j)] + ECc[2 * RC + G.ri(i, j)] + ECc[2 * RC + G.ri(i - 1, j - 1)] +
                 ECc[2 * RC + G.ri(i, j - 1)]));
    return;
  }
  const double *FXm = M.S.fx(q - 1), *FYm = M.S.fy(q - 1), *ECm = M.S.ec(q - 1);
  if (t < nez + nex) {
    const int u = t - nez;
    const int cj = u / G.wx, ci = u - cj * G.wx;
    const int i = G.x0 + ci, j = G.y0 + cj;
    M.S.ex(q)[G.exi(i, j)] =
        (0.5 * (-FYm[7 * NFY + G.fyi(i, j)] - FYc[7 * NFY + G.fyi(i, j)] + FZc[7 * RC + G.ri(i, j - 1)] +
                FZc[7 * RC + G.ri(i, j)]) -
         0.25 * (ECc[G.ri(i, j - 1)] + ECc[G.ri(i, j)] + ECm[G.ri(i, j - 1)] + ECm[G.ri(i, j)]));
  } else {
    const int u = t - nez - nex;
    const int cj = u / (G.wx + 1), ci = u - cj * (G.wx + 1);
    const int i = G.x0 + ci, j = G.y0 + cj;
    M.S.ey(q)[G.eyi(i, j)] =
        (0.5 * (-FZc[6 * RC + G.ri(i - 1, j)] - FZc[6 * RC + G.ri(i, j)] + FXm[7 * NFX + G.fxi(i, j)] +
                FXc[7 * NFX + G.fxi(i, j)]) -
         0.25 * (ECc[RC + G.ri(i - 1, j)] + ECc[RC + G.ri(i, j)] + ECm[RC + G.ri(i - 1, j)] + ECm[RC + G.ri(i, j)]));
  }
}

// Update item t of plane k (godunov.pyx:215-252, ct.pyx:15-123, cons2prim):
// the plane's fluxes, the z fluxes of levels k and k+1, Ez of plane k and
// Ex, Ey of levels k and k+1 are complete.  Returns the new state's CFL
// value (corrector) or 0.
template <int ORDER>
__device__ __forceinline__ double update_item(const March<ORDER>& M, int k, int t, unsigned& e) {
  const Geo& G = M.G;
  const Inst& I = *M.I;
  const int cj = t / G.wx, ci = t - cj * G.wx;
  const int i = G.x0 + ci, j = G.y0 + cj;
  const long long c = k * M.sz + j * M.sy + i;
  const double *FXp = M.S.fx(k), *FYp = M.S.fy(k), *FZp = M.S.fz(k), *FZq = M.S.fz(k + 1);
  const double *EZp = M.S.ez(k), *EXp = M.S.ex(k), *EXq = M.S.ex(k + 1), *EYp = M.S.ey(k), *EYq = M.S.ey(k + 1);
  double w0[NM], un[NM];
  double bxl0, bxr0, byb0, byt0, bzb0, bzt0;
  if constexpr (ORDER == 0) {
    // the stage input, staged through the index maps
    const Plane<0> Wk{M.buf(k)}, Wt{M.buf(k + 1)};
#pragma unroll
    for (int n = 0; n < NM; ++n) w0[n] = Wk(G, n, i, j);
    bxl0 = Wk(G, NM, i, j);
    bxr0 = Wk(G, NM, i + 1, j);
    byb0 = Wk(G, NM + 1, i, j);
    byt0 = Wk(G, NM + 1, i, j + 1);
    bzb0 = Wk(G, NM + 2, i, j);
    bzt0 = Wt(G, NM + 2, i, j);
  } else {
    // w^n and b^n from global memory; faces on the domain boundary through the maps
    const double* __restrict__ wn = I.w[M.parity];
    const double* __restrict__ bnf = I.b[M.parity];
#pragma unroll
    for (int n = 0; n < NM; ++n) w0[n] = wn[n * I.sv + c];
    const bool edge = i == I.ng || i == M.i2 || j == I.ng || j == M.j2 || k == I.ng || k == M.k2;
    if (edge) {
      bxl0 = face_mapped<0>(I, bnf, i, j, k, M.mx, M.my, M.mz);
      bxr0 = face_mapped<0>(I, bnf, i + 1, j, k, M.mx, M.my, M.mz);
      byb0 = face_mapped<1>(I, bnf, i, j, k, M.mx, M.my, M.mz);
      byt0 = face_mapped<1>(I, bnf, i, j + 1, k, M.mx, M.my, M.mz);
      bzb0 = face_mapped<2>(I, bnf, i, j, k, M.mx, M.my, M.mz);
      bzt0 = face_mapped<2>(I, bnf, i, j, k + 1, M.mx, M.my, M.mz);
    } else {
      bxl0 = bnf[c];
      bxr0 = bnf[c + 1];
      byb0 = bnf[I.sv + c];
      byt0 = bnf[I.sv + c + M.sy];
      bzb0 = bnf[2 * I.sv + c];
      bzt0 = bnf[2 * I.sv + c + M.sz];
    }
  }
  prim2cons(un, w0, I.gam);
  const double dt = M.dt;
  const double dx = I.dlf[0][i], dy = I.dlf[1][j], dz = I.dlf[2][k];
#if BNZ_FAST_MATH
  const double idx = I.dlf_inv[0][i], idy = I.dlf_inv[1][j], idz = I.dlf_inv[2][k];
  const double dtdv = dt * idx * idy * idz;
#else
  const double vol = dx * dy * dz;
  const double dtdv = dt / vol;
#endif
  const double dax = dy * dz, day = dx * dz, daz = dx * dy;
  double u[NM];
  const int ql = G.fxi(i, j), qr = G.fxi(i + 1, j), qb = G.fyi(i, j), qt = G.fyi(i, j + 1), qz = G.ri(i, j);
#pragma unroll
  for (int n = 0; n < 6; ++n) {
    double v = un[n] - dtdv * (dax * FXp[n * NFX + qr] - dax * FXp[n * NFX + ql]);
    v -= dtdv * (day * FYp[n * NFY + qt] - day * FYp[n * NFY + qb]);
    v -= dtdv * (daz * FZq[n * RC + qz] - daz * FZp[n * RC + qz]);
    u[n] = v;
  }
  // faces (ct.pyx:15-91): Bx from Ez of the plane and Ey of its two levels,
  // By from Ez and Ex, Bz (levels k and k+1) from Ey and Ex of its level
#if BNZ_FAST_MATH
  double dtda = dt * idy * idz;
#else
  double dtda = dt / (dy * dz);
#endif
  double vxl = bxl0;
  vxl -= dtda * (dz * EZp[G.ezi(i, j + 1)] - dz * EZp[G.ezi(i, j)]);
  vxl += dtda * (dy * EYq[G.eyi(i, j)] - dy * EYp[G.eyi(i, j)]);
  double vxr = bxr0;
  vxr -= dtda * (dz * EZp[G.ezi(i + 1, j + 1)] - dz * EZp[G.ezi(i + 1, j)]);
  vxr += dtda * (dy * EYq[G.eyi(i + 1, j)] - dy * EYp[G.eyi(i + 1, j)]);
#if BNZ_FAST_MATH
  dtda = dt * idx * idz;
#else
  dtda = dt / (dx * dz);
#endif
  double vyb = byb0 + dtda * (dz * EZp[G.ezi(i + 1, j)] - dz * EZp[G.ezi(i, j)]);
  vyb -= dtda * (dx * EXq[G.exi(i, j)] - dx * EXp[G.exi(i, j)]);
  double vyt = byt0 + dtda * (dz * EZp[G.ezi(i + 1, j + 1)] - dz * EZp[G.ezi(i, j + 1)]);
  vyt -= dtda * (dx * EXq[G.exi(i, j + 1)] - dx * EXp[G.exi(i, j + 1)]);
#if BNZ_FAST_MATH
  dtda = dt * idx * idy;
#else
  dtda = dt / (dx * dy);
#endif
  double vzb = bzb0 - dtda * (dy * EYp[G.eyi(i + 1, j)] - dy * EYp[G.eyi(i, j)]);
  vzb += dtda * (dx * EXp[G.exi(i, j + 1)] - dx * EXp[G.exi(i, j)]);
  double vzt = bzt0 - dtda * (dy * EYq[G.eyi(i + 1, j)] - dy * EYq[G.eyi(i, j)]);
  vzt += dtda * (dx * EXq[G.exi(i, j + 1)] - dx * EXq[G.exi(i, j)]);
  // face-to-cell field (ct.pyx:96-123)
  u[BX] = ((I.lv[0][i] - I.lf[0][i]) * vxl + (I.lf[0][i + 1] - I.lv[0][i]) * vxr) * I.dlf_inv[0][i];
  u[BY] = ((I.lv[1][j] - I.lf[1][j]) * vyb + (I.lf[1][j + 1] - I.lv[1][j]) * vyt) * I.dlf_inv[1][j];
  u[BZ] = ((I.lv[2][k] - I.lf[2][k]) * vzb + (I.lf[2][k + 1] - I.lv[2][k]) * vzt) * I.dlf_inv[2][k];
  if (I.src) {
    // integrator.pyx:132-170 add_source_terms, with the stage input's rho and
    // v: w^n in the predictor, ws in the corrector
    double fs[3];
    if (I.fdriv) {
      fs[0] = I.fdriv[c];
      fs[1] = I.fdriv[I.sv + c];
      fs[2] = I.fdriv[2 * I.sv + c];
    }
    const double srho = ORDER ? I.ws[c] : w0[RHO];
    const double svx = ORDER ? I.ws[VX * I.sv + c] : w0[VX];
    const double svy = ORDER ? I.ws[VY * I.sv + c] : w0[VY];
    const double svz = ORDER ? I.ws[VZ * I.sv + c] : w0[VZ];
    const bool grav = I.grav[0] != 0. || I.grav[1] != 0. || I.grav[2] != 0.;
    srcterm::apply(u, srho, svx, svy, svz, I.grav, grav, I.fdriv ? fs : nullptr, dt);
  }
  double wo[NM];
  cons2prim(wo, u, I.gam);
  if (ORDER == 1) e |= plain::check_prim(wo);
  double* __restrict__ wout = ORDER ? I.w[M.parity ^ 1] : I.ws;
  double* __restrict__ bout = ORDER ? I.b[M.parity ^ 1] : I.bs;
#pragma unroll
  for (int n = 0; n < NM; ++n) wout[n * I.sv + c] = wo[n];
  bout[c] = vxl;
  bout[I.sv + c] = vyb;
  bout[2 * I.sv + c] = vzb;
  if (i == M.ilast) bout[c + 1] = vxr;
  if (j == M.jlast) bout[I.sv + c + M.sy] = vyt;
  if (k == M.klast) bout[2 * I.sv + c + M.sz] = vzt;
  if (ORDER == 0) return 0.;
  // the next step's CFL (new_dt.pyx:55-99) on the new state
  const double vf = fms(wo, I.gam);
  const double cx = fabs(wo[VX]) + vf, cy = fabs(wo[VY]) + vf, cz = fabs(wo[VZ]) + vf;
#if BNZ_FAST_MATH
  return fmax(fmax(cx * idx, cy * idy), cz * idz);
#else
  return fmax(fmax(cx / dx, cy / dy), cz / dz);
#endif
}

// The march of one chunk.  ORDER 0: predictor, ORDER 1: corrector.
// Per plane q: the flux items of plane q (and the z faces of level q), then
// the edge items, then -- in one phase -- the update of plane q-1 together
// with the pre-flux items of plane q+1 (slopes, E_c), which touch disjoint
// slots: three barriers per plane, and the update's threads share the phase
// with the next plane's work.
template <int ORDER, int RS, int LIM>
__global__ void __launch_bounds__(NT, 1) k_vl3d(const Inst* __restrict__ insts, const Tile* __restrict__ tiles,
                                                int parity, int cp, const unsigned char* __restrict__ maps) {
  extern __shared__ __align__(128) double smem_raw[];
  __shared__ Inst sI;
  __shared__ __align__(8) unsigned long long bar[4];
  __shared__ int s_fail;
  double* sm = smem_raw + ((128u - (fused::tma::saddr(smem_raw) & 127u)) & 127u) / sizeof(double);
  const Tile T = tiles[blockIdx.x];
  {
    constexpr int NW = sizeof(Inst) / sizeof(int);
    static_assert(sizeof(Inst) % sizeof(int) == 0, "Inst must be int-aligned");
    const int* src = reinterpret_cast<const int*>(insts + T.inst);
    int* dst = reinterpret_cast<int*>(&sI);
    for (int t = threadIdx.x; t < NW; t += NT) dst[t] = src[t];
    if (threadIdx.x == 0) s_fail = 0;
  }
  __syncthreads();
  const Inst& I = sI;
  const double dtf = I.ds->dt;
  const long long sy = I.nx, sz = (long long)I.nx * I.ny;
  if (!(dtf > 0.)) {
    if (ORDER == 1) {
      // time has reached tmax: carry the chunk's state over unchanged
      const double* w = I.w[parity];
      const double* b = I.b[parity];
      double* w1 = I.w[parity ^ 1];
      double* b1 = I.b[parity ^ 1];
      const int i2 = I.ng + I.N[0] - 1, j2 = I.ng + I.N[1] - 1, k2 = I.ng + I.N[2] - 1;
      for (int t = threadIdx.x; t < T.wx * T.wy * T.wz; t += NT) {
        const int i = T.x0 + t % T.wx, j = T.y0 + (t / T.wx) % T.wy, k = T.z0 + t / (T.wx * T.wy);
        const long long c = k * sz + j * sy + i;
#pragma unroll
        for (int n = 0; n < NM; ++n) w1[n * I.sv + c] = w[n * I.sv + c];
        for (int n = 0; n < 3; ++n) b1[n * I.sv + c] = b[n * I.sv + c];
        if (i == i2) b1[c + 1] = b[c + 1];
        if (j == j2) b1[I.sv + c + sy] = b[I.sv + c + sy];
        if (k == k2) b1[2 * I.sv + c + sz] = b[2 * I.sv + c + sz];
      }
    }
    return;
  }
  March<ORDER> M;
  M.I = &I;
  M.S.set(sm);
  M.G.x0 = T.x0;
  M.G.y0 = T.y0;
  M.G.wx = T.wx;
  M.G.wy = T.wy;
  M.G.xs = (T.x0 - 2) & ~1;
  M.G.ys = T.y0 - 2;
  M.parity = parity;
  M.cp = cp;
  M.dt = ORDER == 0 ? 0.5 * dtf : dtf;
  M.mx = axis_map3(I, 0);
  M.my = axis_map3(I, 1);
  M.mz = axis_map3(I, 2);
  M.i2 = I.ng + I.N[0] - 1;
  M.j2 = I.ng + I.N[1] - 1;
  M.k2 = I.ng + I.N[2] - 1;
  M.ilast = ORDER ? M.i2 : I.nx - 2;
  M.jlast = ORDER ? M.j2 : I.ny - 2;
  M.klast = ORDER ? M.k2 : I.nz - 2;
  M.sy = sy;
  M.sz = sz;
  const Geo& G = M.G;
  const int zlo = T.z0 - 1, zhi = T.z0 + T.wz;  // planes q = zlo .. zhi; updates of z0 .. z0+wz-1
  M.pbase = ORDER ? T.z0 - 2 : T.z0 - 1;        // first staged plane
  const int pbase = M.pbase;
  const int plast = ORDER ? zhi + 1 : zhi;      // last staged plane
  const bool tma_on = ORDER == 1 && T.tma && maps;
  const void* map = tma_on ? (const void*)(maps + (size_t)T.inst * 128) : nullptr;
  // stage plane p into its ring buffer (one thread issues the TMA box; all
  // threads issue cp.async and commit one group, an empty one past plast)
  auto issue = [&](int p) {
    if (p > plast) {
      if (!tma_on) cp_async_commit();
      return;
    }
    if (ORDER == 0) {
      stage_pred_plane(I, G, p, I.w[parity], I.b[parity], M.buf(p));
      cp_async_commit();
    } else if (tma_on) {
      if (threadIdx.x == 0) {
        unsigned long long* b = &bar[(p - pbase) & 3];
        fused::tma::fence_async_shared();
        fused::tma::arrive_expect(b, BOX_BYTES);
        load_4d(M.buf(p), b, map, G.xs, G.ys, p, 0);
      }
    } else {
      stage_ws_plane(I, G, p, M.buf(p));
      cp_async_commit();
    }
  };
  // every thread observes plane p's TMA phase (bounded); cp.async: all but the
  // newest group are complete
  auto ready = [&](int p) {
    if (tma_on) {
      if (!fused::tma::wait(&bar[(p - pbase) & 3], (unsigned)((p - pbase) >> 2) & 1u)) s_fail = 1;
    } else {
      cp_async_wait1();
    }
  };
  if (tma_on && threadIdx.x == 0) {
    for (int b = 0; b < 4; ++b) fused::tma::bar_init(&bar[b], 1);
    fused::tma::fence_bar_init();
    fused::tma::prefetch_map(map);
  }
  __syncthreads();
  // prologue: the planes of the first pre-flux phase, and one ahead
  int issued, waited;
  if (ORDER == 1) {
    issue(pbase);      // zlo - 1
    issue(pbase + 1);  // zlo
    issue(pbase + 2);  // zlo + 1
    issue(pbase + 3);  // zlo + 2
    if (tma_on) {
      ready(pbase);
      ready(pbase + 1);
      ready(pbase + 2);
    } else {
      cp_async_wait1();
    }
    issued = pbase + 3;
    waited = pbase + 2;
  } else {
    issue(pbase);      // zlo
    issue(pbase + 1);  // zlo + 1
    cp_async_wait1();
    issued = pbase + 1;
    waited = pbase;
  }
  __syncthreads();
  for (int u = threadIdx.x; u < npre(M); u += NT) pre_item<ORDER, LIM>(M, zlo, u);
  __syncthreads();
  unsigned e = 0;
  double cmax = 0.;
  const int nfx = (G.wx + 1) * (G.wy + 2), nfy = (G.wx + 2) * (G.wy + 1), nc = (G.wx + 2) * (G.wy + 2);
  const int nez = (G.wx + 1) * (G.wy + 1), nexy = G.wx * (G.wy + 1) + (G.wx + 1) * G.wy;
  const int ncell = G.wx * G.wy;
  for (int q = zlo; q <= zhi; ++q) {
    const bool first = q == zlo;
    if (ORDER == 0) {
      issue(q + 2);  // into the buffer of plane q-2 (last read before the previous barrier)
      issued = q + 2;
    }
    // --- fluxes of plane q and the z faces of level q ---
    {
      const int nf = nfx + nfy + (first ? 0 : nc);
      for (int t = threadIdx.x; t < nf; t += NT) flux_item<ORDER, RS>(M, q, t, nfx, nfy, e);
    }
    __syncthreads();
    if (ORDER == 1) {
      issue(q + 3);  // into the buffer of plane q-1: its last reader was the z-face phase above
      issued = q + 3;
    }
    // --- edge EMFs: Ez of plane q, Ex / Ey of level q ---
    {
      const int ne = nez + (first ? 0 : nexy);
      for (int t = threadIdx.x; t < ne; t += NT) edge_item(M, q, t, nez, G.wx * (G.wy + 1));
    }
    // the plane the next pre-flux phase reads last
    const int need = ORDER ? q + 2 : q + 1;
    if (need <= plast) {
      ready(need);
      waited = need;
    }
    __syncthreads();
    if (s_fail) break;
    // --- the update of plane q-1 and the pre-flux items of plane q+1 ---
    {
      const int nu = (!first && q - 1 >= T.z0) ? ncell : 0;
      const int np = q + 1 <= zhi ? npre(M) : 0;
      for (int t = threadIdx.x; t < np + nu; t += NT) {
        if (t < np) {
          pre_item<ORDER, LIM>(M, q + 1, t);
        } else {
          const double c = update_item<ORDER>(M, q - 1, t - np, e);
          if (c > cmax) cmax = c;
        }
      }
    }
    __syncthreads();  // the plane's slots and buffers are free
  }
  if (s_fail) {
    // a staged plane did not arrive: flag it, give the loads still in flight a
    // bounded wait, and leave without writing the rest of the chunk
    if (threadIdx.x == 0) {
      atomicOr(I.err, (unsigned)ERR_TIMEOUT);
      for (int p = waited + 1; p <= issued && p <= plast; ++p)
        fused::tma::wait(&bar[(p - pbase) & 3], (unsigned)((p - pbase) >> 2) & 1u);
    }
    return;
  }
  if (!tma_on) cp_async_wait0();
  if (ORDER == 1) {
    for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    if ((threadIdx.x & 31) == 0 && cmax > 0.)
      atomicMax(&I.ds->cds_bits[parity ^ 1], (unsigned long long)__double_as_longlong(cmax));
  }
  if (e) atomicOr(I.err, e);
}

// CFL maximum of the current state into slot `parity` (new_dt.pyx:18-135),
// over the corrector chunks (the active cells).
__global__ void k_cds3(const Inst* __restrict__ insts, const Tile* __restrict__ tiles, int parity) {
  __shared__ double red[32];
  const Tile T = tiles[blockIdx.x];
  const Inst& I = insts[T.inst];
  const double* w = I.w[parity];
  double cmax = 0.;
  for (int t = threadIdx.x; t < T.wx * T.wy * T.wz; t += blockDim.x) {
    const int i = T.x0 + t % T.wx, j = T.y0 + (t / T.wx) % T.wy, k = T.z0 + t / (T.wx * T.wy);
    const long long c = ((long long)k * I.ny + j) * I.nx + i;
    double ww[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) ww[n] = w[n * I.sv + c];
    const double vf = fms(ww, I.gam);
    const double cx = fabs(ww[VX]) + vf, cy = fabs(ww[VY]) + vf, cz = fabs(ww[VZ]) + vf;
    const double cds = fmax(fmax(cx / I.dlf[0][i], cy / I.dlf[1][j]), cz / I.dlf[2][k]);
    if (cds > cmax) cmax = cds;
  }
  for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = cmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) m = fmax(m, red[q]);
    if (m > 0.) atomicMax(&I.ds->cds_bits[parity], (unsigned long long)__double_as_longlong(m));
  }
}

}  // namespace fused3
