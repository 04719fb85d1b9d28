// bnz_fused.cuh -- fused tile kernels of the 2D VL2 step (predictor, corrector)
// and their batched launch over many independent grids.
//
// One step is three launches for the whole batch:
//   k_dt_batch  per-instance CFL dt = cour / max(|v|+c_f)/dx (+ tmax clip),
//               from the max the previous corrector accumulated;
//   k_pred2d    predictor (vanleer.pyx:104-120): per tile, donor-cell HLLD
//               fluxes -> shared memory, CT corner EMFs -> shared memory, then
//               per cell the half-step conserved update, the half-step faces
//               and cons2prim; writes ws (9) and bs (3) on the predictor range
//               (cells 1..Ntot-2 of every active axis);
//   k_corr2d    corrector (vanleer.pyx:130-151): per active tile, PLM + HLLD
//               fluxes from ws/bs, EMFs, the full-step update of u^n and B^n,
//               cons2prim; writes the new prim and face field, and reduces the
//               next step's CFL max into the instance's slot.
// k_pred2d_pq / k_corr2d_pq are the same two stages as persistent kernels:
// one resident grid per launch takes tiles from a work queue and loads the
// next tile's inputs by TMA (cp.async.bulk.tensor, mbarrier-completed) into
// the second of two shared-memory buffers while the current tile computes.
// u^n is rebuilt as prim2cons(w^n), which is bitwise what the reference keeps
// in its cons array between steps (vanleer.pyx:163).  Ghost values are never
// stored: loads outside the active range go through the boundary-condition
// index map (the source index and sign grid_bc_funcs.pyx / util_bc.pyx would
// copy), so no ghost-fill pass runs between steps.
// Included inside the per-floating-point-mode namespace.
#pragma once

namespace fused {

using namespace dev;

using Inst = FusedInst;
using Tile = FusedTile;

// ---------------------------------------------------------------------------
// boundary-condition index maps (grid_bc_funcs.pyx:36-330, util_bc.pyx)
// ---------------------------------------------------------------------------

struct AxisMap {
  int a1, a2, n, f0, f1, face_aware;
};

__device__ __forceinline__ AxisMap axis_map(const Inst& I, int ax) {
  AxisMap m;
  m.a1 = I.ng;
  m.a2 = I.ng + I.N[ax] - 1;
  m.n = I.N[ax];
  m.f0 = I.bc[ax][0];
  m.f1 = I.bc[ax][1];
  m.face_aware = I.face_aware;
  return m;
}

// cell-centred along this axis: source index, sign flips for the normal component
__device__ __forceinline__ int map_cell(int a, const AxisMap& m, bool& flip) {
  flip = false;
  if (a < m.a1) {
    if (m.f0 == 0) return a + m.n;
    if (m.f0 == 1) return m.a1;
    flip = true;
    return 2 * m.a1 - 1 - a;
  }
  if (a > m.a2) {
    if (m.f1 == 0) return a - m.n;
    if (m.f1 == 1) return m.a2;
    flip = true;
    return 2 * m.a2 + 1 - a;
  }
  return a;
}

// face-centred along this axis (the face normal to it)
__device__ __forceinline__ int map_face(int a, const AxisMap& m, bool& flip, bool& zero) {
  flip = false;
  zero = false;
  if (a < m.a1) {
    if (m.f0 == 0) return a + m.n;
    if (m.f0 == 1) return m.a1;
    flip = true;
    return 2 * m.a1 - a;
  }
  if (a == m.a1 && m.f0 == 2) {
    zero = true;
    return a;
  }
  if (a > m.a2) {
    if (m.f1 == 0) return a - m.n;
    if (m.f1 == 1) {
      if (!m.face_aware) return m.a2;
      return a == m.a2 + 1 ? a : m.a2 + 1;
    }
    if (a == m.a2 + 1) {
      zero = true;
      return a;
    }
    flip = true;
    return 2 * m.a2 + 2 - a;
  }
  return a;
}

// prim at cell (i, j) with ghost indices mapped
__device__ __forceinline__ void load_prim_all(const Inst& I, const double* __restrict__ w, int i, int j,
                                              const AxisMap& mx, const AxisMap& my, bool interior, double* out) {
  bool fx = false, fy = false;
  int si = i, sj = j;
  if (!interior) {
    si = map_cell(i, mx, fx);
    sj = map_cell(j, my, fy);
  }
  const long long c = (long long)sj * I.nx + si;
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    double v = w[n * I.sv + c];
    if ((fx && (n == VX || n == BX)) || (fy && (n == VY || n == BY))) v = -v;
    out[n] = v;
  }
}

// face component COMP at (i, j) with ghost indices mapped
template <int COMP>
__device__ __forceinline__ double load_face(const Inst& I, const double* __restrict__ b, int i, int j,
                                            const AxisMap& mx, const AxisMap& my, bool interior) {
  if (interior) return b[COMP * I.sv + (long long)j * I.nx + i];
  bool f1 = false, f2 = false, z1 = false, z2 = false;
  int si, sj;
  if (COMP == 0) {
    si = map_face(i, mx, f1, z1);
    sj = map_cell(j, my, f2);
    f2 = false;  // tangential along y
  } else if (COMP == 1) {
    si = map_cell(i, mx, f1);
    f1 = false;
    sj = map_face(j, my, f2, z2);
  } else {
    si = map_cell(i, mx, f1);
    sj = map_cell(j, my, f2);
    f1 = f2 = false;
  }
  if (z1 || z2) return 0.;
  double v = b[COMP * I.sv + (long long)sj * I.nx + si];
  return (f1 != f2) ? -v : v;
}

// ---------------------------------------------------------------------------
// shared-memory layout of one tile
// ---------------------------------------------------------------------------

constexpr int NF = 8;  // stored flux values: 6 hydro + 2 field (for the EMFs)

struct Layout {
  int wx, wy;
  int nfx, nfy, nec, nee;
  int sfx, sfy;  // field strides of the x / y flux arrays (their allocated sizes)
  __device__ __forceinline__ void set(int wx_, int wy_) {
    wx = wx_;
    wy = wy_;
    nfx = (wx + 1) * (wy + 2);
    nfy = (wx + 2) * (wy + 1);
    nec = (wx + 2) * (wy + 2);
    nee = (wx + 1) * (wy + 1);
    sfx = nfx;
    sfy = nfy;
  }
  // the tile's arrays laid out for the largest tile TXM x TYM: compile-time
  // field strides, whatever the tile's own size
  template <int TXM, int TYM>
  __device__ __forceinline__ void set_max(int wx_, int wy_) {
    set(wx_, wy_);
    sfx = (TXM + 1) * (TYM + 2);
    sfy = (TXM + 2) * (TYM + 1);
  }
  // x faces i = x0..x0+wx, rows j = y0-1..y0+wy
  __device__ __forceinline__ int fx(int fi, int fj) const { return (fj + 1) * (wx + 1) + fi; }
  // y faces j = y0..y0+wy, columns i = x0-1..x0+wx
  __device__ __forceinline__ int fy(int fi, int fj) const { return fj * (wx + 2) + fi + 1; }
  // cells i = x0-1..x0+wx, j = y0-1..y0+wy
  __device__ __forceinline__ int ec(int ci, int cj) const { return (cj + 1) * (wx + 2) + ci + 1; }
  // corners i = x0..x0+wx, j = y0..y0+wy
  __device__ __forceinline__ int ee(int ci, int cj) const { return cj * (wx + 1) + ci; }
};

template <int TXM, int TYM, int RING>
struct Smem {
  static constexpr int NFX = (TXM + 1) * (TYM + 2);
  static constexpr int NFY = (TXM + 2) * (TYM + 1);
  static constexpr int NEC = (TXM + 2) * (TYM + 2);
  static constexpr int NEE = (TXM + 1) * (TYM + 1);
  static constexpr int NSW = RING ? NM * (TXM + 2 * RING) * (TYM + 2 * RING) : 0;  // staged cells
  static constexpr int NSD = RING == 2 ? 8 * (TXM + 2) * (TYM + 2) : 0;              // corrector slopes
  static constexpr size_t bytes = sizeof(double) * ((size_t)NF * (NFX + NFY) + NEC + NEE + NSW + NSD);
};

// ---------------------------------------------------------------------------
// Stage 0: the tile's input cells into shared memory in one coalesced pass.
// Predictor: w^n on the tile plus one ring, ghost indices through the BC map.
// Corrector: ws on the tile plus two rings (the predictor wrote those cells).
// ---------------------------------------------------------------------------

// t / d for small t (t * d < 2^32) by a multiply-high with m = ceil(2^32 / d);
// d = 1 (m would need 33 bits) is handled separately.
struct FastDiv {
  unsigned d, m;
  __device__ __forceinline__ void set(unsigned dd) {
    d = dd;
    m = dd > 1u ? 0xFFFFFFFFu / dd + 1u : 0u;
  }
  __device__ __forceinline__ unsigned div(unsigned t) const { return d > 1u ? __umulhi(t, m) : t; }
};

struct Stage {
  int x0, y0, w, h;  // region origin (array coordinates) and size
  __device__ __forceinline__ int at(int n, int i, int j) const { return (n * h + (j - y0)) * w + (i - x0); }
  __device__ __forceinline__ int cells() const { return w * h; }
};

template <bool MAP>
__device__ __forceinline__ void stage_cells(const Inst& I, const double* __restrict__ src, const Stage& S, double* sW) {
  const AxisMap mx = axis_map(I, 0), my = axis_map(I, 1);
  FastDiv dw;
  dw.set(S.w);
  for (int t = threadIdx.x; t < S.cells(); t += blockDim.x) {
    const int cj = dw.div(t), ci = t - cj * S.w;
    int i = S.x0 + ci, j = S.y0 + cj;
    bool fx = false, fy = false;
    if (MAP) {
      i = map_cell(i, mx, fx);
      j = map_cell(j, my, fy);
    }
    const long long c = (long long)j * I.nx + i;
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      double v = src[n * I.sv + c];
      if (MAP && ((fx && (n == VX || n == BX)) || (fy && (n == VY || n == BY)))) v = -v;
      sW[n * S.cells() + t] = v;
    }
  }
}

// The cells of region R (no ghost mapping) into shared memory laid out as S
// (a larger region with fixed sizes): the plain-load counterpart of a TMA box.
__device__ __forceinline__ void stage_cells_into(const Inst& I, const double* __restrict__ src, const Stage& R,
                                                 const Stage& S, double* sW) {
  FastDiv dw;
  dw.set(R.w);
  for (int t = threadIdx.x; t < R.cells(); t += blockDim.x) {
    const int cj = dw.div(t), ci = t - cj * R.w;
    const int i = R.x0 + ci, j = R.y0 + cj;
    const long long c = (long long)j * I.nx + i;
    const int d = S.at(0, i, j);
#pragma unroll
    for (int n = 0; n < NM; ++n) sW[n * S.cells() + d] = src[n * I.sv + c];
  }
}

// Cell readers for the flux stage: staged shared memory, or global memory
// with the BC map applied on the fly.
struct SmemCells {
  const double* sW;
  Stage S;
  int nc;
  __device__ __forceinline__ double get(int n, int i, int j) const { return sW[n * nc + S.at(0, i, j)]; }
  // value at (i, j) shifted by `o` cells along the axis with stride `st` (1: x, S.w: y)
  __device__ __forceinline__ const double* ptr(int n, int i, int j) const { return sW + n * nc + S.at(0, i, j); }
  __device__ __forceinline__ int stride(int ax) const { return ax == 0 ? 1 : S.w; }
  __device__ __forceinline__ void load_all(int i, int j, double* out) const {
    const int c = S.at(0, i, j);
#pragma unroll
    for (int n = 0; n < NM; ++n) out[n] = sW[n * nc + c];
  }
};

struct GlobalCells {
  const Inst* I;
  const double* w;
  AxisMap mx, my;
  bool interior;
  __device__ __forceinline__ double get(int n, int i, int j) const {
    if (interior) return w[n * I->sv + (long long)j * I->nx + i];
    bool fx, fy;
    const int si = map_cell(i, mx, fx), sj = map_cell(j, my, fy);
    double v = w[n * I->sv + (long long)sj * I->nx + si];
    return ((fx && (n == VX || n == BX)) || (fy && (n == VY || n == BY))) ? -v : v;
  }
  __device__ __forceinline__ void load_all(int i, int j, double* out) const {
    load_prim_all(*I, w, i, j, mx, my, interior, out);
  }
};

// Face readers of the predictor: global memory through the BC map, or the
// faces a persistent predictor staged in shared memory (interior tiles).
struct GlobalFaces {
  const Inst* I;
  const double* b;
  AxisMap mx, my;
  bool interior;
  template <int COMP>
  __device__ __forceinline__ double get(int i, int j) const {
    return load_face<COMP>(*I, b, i, j, mx, my, interior);
  }
};

struct SmemFaces {
  const double* sB;
  Stage S;
  template <int COMP>
  __device__ __forceinline__ double get(int i, int j) const {
    return sB[COMP * S.cells() + S.at(0, i, j)];
  }
};

// ---------------------------------------------------------------------------
// Stage 1 of the predictor: donor-cell interface fluxes and the cell-centred
// EMF.  (The corrector's PLM flux stage is stage_fluxes_plm below.)
// ---------------------------------------------------------------------------

template <int RS, class Cells, class Faces>
__device__ __forceinline__ void stage_fluxes(const Inst& I, const Tile& T, const Layout& L, const Cells& W,
                                             const Faces& F, double* sFX, double* sFY, double* sEC,
                                             unsigned& err) {
  // every face is one item; the first nec items also form one cell's E_c
  // (nec <= nfx + nfy for any tile), so the loop is faces-only in length
  const int total = L.nfx + L.nfy;
  FastDiv dx1, dx2;
  dx1.set(L.wx + 1);
  dx2.set(L.wx + 2);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    if (t < L.nec) {
      // cell-centred E_z = -(vx by - vy bx) (ct.pyx:148) of cell slot t
      const int q = dx2.div(t);
      const int ci = t - q * (L.wx + 2) - 1, cj = q - 1;
      const int i = T.x0 + ci, j = T.y0 + cj;
      const double vx = W.get(VX, i, j), vy = W.get(VY, i, j), bxc = W.get(BX, i, j), byc = W.get(BY, i, j);
      sEC[L.ec(ci, cj)] = -(vx * byc - vy * bxc);
    }
    // one Riemann call site for both directions: the face's cells and normal
    // field are gathered per direction, the flux stored per direction
    const bool xf = t < L.nfx;
    int i, j, di, dj, qq;
    if (xf) {
      // x face at column i (between cells i-1 and i), row j
      const int q = dx1.div(t);
      const int fi = t - q * (L.wx + 1), fj = q - 1;
      i = T.x0 + fi;
      j = T.y0 + fj;
      di = 1;
      dj = 0;
      qq = L.fx(fi, fj);
    } else {
      // y face at row j (between cells j-1 and j), column i; sweep frame AX = 1
      const int u = t - L.nfx;
      const int q = dx2.div(u);
      const int fi = u - q * (L.wx + 2) - 1, fj = q;
      i = T.x0 + fi;
      j = T.y0 + fj;
      di = 0;
      dj = 1;
      qq = L.fy(fi, fj);
    }
    double wL[NM], wR[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      if (n == BX) continue;
      const int gv = xf ? n : plain::perm<1>(n);
      wL[n] = W.get(gv, i - di, j - dj);
      wR[n] = W.get(gv, i, j);
    }
    wL[BX] = wR[BX] = xf ? F.template get<0>(i, j) : F.template get<1>(i, j);
    double f[NM];
    riemann<RS, true>(f, wL, wR, I.gam, err);
    if (xf) {
#pragma unroll
      for (int n = 0; n < 6; ++n) sFX[n * L.sfx + qq] = f[n];
      sFX[6 * L.sfx + qq] = f[BY];  // fx[BY]
      sFX[7 * L.sfx + qq] = f[BZ];  // fx[BZ]
    } else {
      // local -> global (godunov.pyx:297-324 for the y sweep)
      sFY[0 * L.sfy + qq] = f[RHO];
      sFY[1 * L.sfy + qq] = f[VZ];   // global MX
      sFY[2 * L.sfy + qq] = f[VX];   // global MY
      sFY[3 * L.sfy + qq] = f[VY];   // global MZ
      sFY[4 * L.sfy + qq] = f[EN];
      sFY[5 * L.sfy + qq] = f[PSC];
      sFY[6 * L.sfy + qq] = f[BZ];   // fy[BX]
      sFY[7 * L.sfy + qq] = f[BY];   // fy[BZ]
    }
  }
}

// Corrector flux stage with the PLM slopes formed once per cell: for each
// direction, half slopes d = 0.5 lim(w - w_-, w_+ - w) of the 8 swept variables
// go to shared memory (cells x0-1..x0+wx, y0-1..y0+wy), then each face takes
// wL = w(i-1) + d(i-1), wR = w(i) - d(i) -- the same values reconstr_linear
// forms per face (reconstr_c.c:54-91), with half the limiter evaluations.
struct SlopeBuf {
  double* d;  // 8 fields of s doubles, the cells (wx+2) x (wy+2) first in each
  int w, n;   // row width (wx+2), cells
  int s;      // field stride
  int x0, y0; // array coordinates of the first cell (x0-1, y0-1)
  __device__ __forceinline__ int at(int i, int j) const { return (j - y0) * w + (i - x0); }
};

__device__ __forceinline__ int slot8(int n) { return n < BX ? n : n - 1; }

// cp (charact_proj): the nine local variables are limited in characteristic
// variables of the cell (reconstr_c.c:54-91 with prim2char / char2prim).
// sEC (x direction only, else null): the cell-centred E_z of the same cells,
// -(vx by - vy bx) (ct.pyx:148); a cell's slot t is its E_c slot too.
template <int AX, int LIM>
__device__ __forceinline__ void stage_slopes(const Layout& L, const SmemCells& W, const SlopeBuf& D, int cp,
                                             double gam, double* sEC) {
  FastDiv dw;
  dw.set(D.w);
  const int st = W.stride(AX);
  for (int t = threadIdx.x; t < D.n; t += blockDim.x) {
    const int cj = dw.div(t), ci = t - cj * D.w;
    const int i = D.x0 + ci, j = D.y0 + cj;
    if (AX == 0 && sEC) {
      const double vx = W.get(VX, i, j), vy = W.get(VY, i, j), bxc = W.get(BX, i, j), byc = W.get(BY, i, j);
      sEC[t] = -(vx * byc - vy * bxc);
    }
    if (cp) {
      double wm[NM], wc[NM], wp[NM], d[NM];
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        const double* a = W.ptr(plain::perm<AX>(n), i, j);
        wm[n] = a[-st];
        wc[n] = a[0];
        wp[n] = a[st];
      }
      half_slopes_char<LIM>(wm, wc, wp, gam, d);
#pragma unroll
      for (int n = 0; n < NM; ++n)
        if (n != BX) D.d[slot8(n) * D.s + t] = d[n];
    } else {
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        if (n == BX) continue;
        const double* a = W.ptr(plain::perm<AX>(n), i, j);
        D.d[slot8(n) * D.s + t] = half_slope<LIM>(a[-st], a[0], a[st]);
      }
    }
  }
}

// SMAX: the slope buffer's field stride (its allocated cells per field), 0
// for the tile's own cell count.
template <int LIM, int RS, int SMAX = 0>
__device__ __forceinline__ void stage_fluxes_plm(const Inst& I, const Tile& T, const Layout& L, const SmemCells& W,
                                                 const double* __restrict__ b, double* sFX, double* sFY, double* sEC,
                                                 double* sD, int cp, unsigned& err) {
  SlopeBuf D;
  D.d = sD;
  D.w = L.wx + 2;
  D.n = (L.wx + 2) * (L.wy + 2);
  D.s = SMAX > 0 ? SMAX : D.n;
  D.x0 = T.x0 - 1;
  D.y0 = T.y0 - 1;
  // x direction: slopes (and E_c), then x faces i = x0..x0+wx on rows y0-1..y0+wy
  stage_slopes<0, LIM>(L, W, D, cp, I.gam, sEC);
  __syncthreads();
  {
    FastDiv dx1;
    dx1.set(L.wx + 1);
    for (int t = threadIdx.x; t < L.nfx; t += blockDim.x) {
      const int q = dx1.div(t);
      const int fi = t - q * (L.wx + 1), fj = q - 1;
      const int i = T.x0 + fi, j = T.y0 + fj;
      const int cl = D.at(i - 1, j), cr = D.at(i, j);
      double wL[NM], wR[NM];
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        if (n == BX) continue;
        wL[n] = W.get(n, i - 1, j) + D.d[slot8(n) * D.s + cl];
        wR[n] = W.get(n, i, j) - D.d[slot8(n) * D.s + cr];
      }
      wL[BX] = wR[BX] = b[(long long)j * I.nx + i];
      double f[NM];
      riemann<RS, true>(f, wL, wR, I.gam, err);
      const int qq = L.fx(fi, fj);
#pragma unroll
      for (int n = 0; n < 6; ++n) sFX[n * L.sfx + qq] = f[n];
      sFX[6 * L.sfx + qq] = f[BY];  // fx[BY]
      sFX[7 * L.sfx + qq] = f[BZ];  // fx[BZ]
    }
  }
  __syncthreads();
  // y direction: slopes, then y faces j = y0..y0+wy on columns x0-1..x0+wx
  stage_slopes<1, LIM>(L, W, D, cp, I.gam, nullptr);
  __syncthreads();
  {
    FastDiv dx2;
    dx2.set(L.wx + 2);
    for (int t = threadIdx.x; t < L.nfy; t += blockDim.x) {
      const int q = dx2.div(t);
      const int fi = t - q * (L.wx + 2) - 1, fj = q;
      const int i = T.x0 + fi, j = T.y0 + fj;
      const int cl = D.at(i, j - 1), cr = D.at(i, j);
      double wL[NM], wR[NM];
#pragma unroll
      for (int n = 0; n < NM; ++n) {
        if (n == BX) continue;
        const int gv = plain::perm<1>(n);
        wL[n] = W.get(gv, i, j - 1) + D.d[slot8(n) * D.s + cl];
        wR[n] = W.get(gv, i, j) - D.d[slot8(n) * D.s + cr];
      }
      wL[BX] = wR[BX] = b[I.sv + (long long)j * I.nx + i];
      double f[NM];
      riemann<RS, true>(f, wL, wR, I.gam, err);
      const int qq = L.fy(fi, fj);
      sFY[0 * L.sfy + qq] = f[RHO];
      sFY[1 * L.sfy + qq] = f[VZ];   // global MX
      sFY[2 * L.sfy + qq] = f[VX];   // global MY
      sFY[3 * L.sfy + qq] = f[VY];   // global MZ
      sFY[4 * L.sfy + qq] = f[EN];
      sFY[5 * L.sfy + qq] = f[PSC];
      sFY[6 * L.sfy + qq] = f[BZ];   // fy[BX]
      sFY[7 * L.sfy + qq] = f[BY];   // fy[BZ]
    }
  }
}

// corner E_z (ct.pyx:204-207)
__device__ __forceinline__ void stage_emf(const Layout& L, const double* sFX, const double* sFY, const double* sEC,
                                          double* sEE) {
  FastDiv dw;
  dw.set(L.wx + 1);
  for (int t = threadIdx.x; t < L.nee; t += blockDim.x) {
    const int cj = dw.div(t), ci = t - cj * (L.wx + 1);
    sEE[t] = (0.5 * (-sFX[6 * L.sfx + L.fx(ci, cj - 1)] - sFX[6 * L.sfx + L.fx(ci, cj)] +
                     sFY[6 * L.sfy + L.fy(ci - 1, cj)] + sFY[6 * L.sfy + L.fy(ci, cj)]) -
              0.25 * (sEC[L.ec(ci - 1, cj)] + sEC[L.ec(ci, cj)] + sEC[L.ec(ci - 1, cj - 1)] + sEC[L.ec(ci, cj - 1)]));
  }
}

// Stage 3: per cell, the conserved update (godunov.pyx:215-252), the face
// update (ct.pyx:15-91), face-to-cell B (ct.pyx:96-123) and cons2prim.
// Returns the new primitive state and the cell's four (five) new faces.
struct CellOut {
  double w[NM];
  double bxl, bxr, byb, byt, bz;
};

// w0: the stage input's prim at the cell (rho, vx, vy, vz used by the source terms)
__device__ __forceinline__ void stage_cell(const Inst& I, const Layout& L, const Tile& T, int ci, int cj,
                                           const double* un, const double* w0, double bxl0, double bxr0,
                                           double byb0, double byt0, double bz0, const double* sFX,
                                           const double* sFY, const double* sEE, double dt, CellOut& o) {
  const int i = T.x0 + ci, j = T.y0 + cj;
  const double dx = I.dlf[0][i], dy = I.dlf[1][j], dz = I.dlf2;
#if BNZ_FAST_MATH
  const double idx = I.dlf_inv[0][i], idy = I.dlf_inv[1][j], idz = 1. / dz;
  double dtdv = dt * idx * idy * idz;
#else
  double vol = dx * dy * dz;
  double dtdv = dt / vol;
#endif
  double dax = dy * dz;
  double day = dx * dz;
  double u[NM];
  const int ql = L.fx(ci, cj), qr = L.fx(ci + 1, cj);
  const int qb = L.fy(ci, cj), qt = L.fy(ci, cj + 1);
#pragma unroll
  for (int n = 0; n < 6; ++n) {
    double v = un[n] - dtdv * (dax * sFX[n * L.sfx + qr] - dax * sFX[n * L.sfx + ql]);
    v -= dtdv * (day * sFY[n * L.sfy + qt] - day * sFY[n * L.sfy + qb]);
    u[n] = v;
  }
  // faces (2D: E_z at corners, E_y = fx[BZ] on x faces, E_x = -fy[BZ] on y faces)
  const double e00 = sEE[L.ee(ci, cj)], e10 = sEE[L.ee(ci + 1, cj)];
  const double e01 = sEE[L.ee(ci, cj + 1)], e11 = sEE[L.ee(ci + 1, cj + 1)];
#if BNZ_FAST_MATH
  double dtda = dt * idy * idz;
#else
  double dtda = dt / (dy * dz);
#endif
  o.bxl = bxl0 - dtda * (dz * e01 - dz * e00);
  o.bxr = bxr0 - dtda * (dz * e11 - dz * e10);
#if BNZ_FAST_MATH
  dtda = dt * idx * idz;
#else
  dtda = dt / (dx * dz);
#endif
  o.byb = byb0 + dtda * (dz * e10 - dz * e00);
  o.byt = byt0 + dtda * (dz * e11 - dz * e01);
#if BNZ_FAST_MATH
  dtda = dt * idx * idy;
#else
  dtda = dt / (dx * dy);
#endif
  const double eyl = sFX[7 * L.sfx + ql], eyr = sFX[7 * L.sfx + qr];
  const double exb = -sFY[7 * L.sfy + qb], ext = -sFY[7 * L.sfy + qt];
  double bz = bz0 - dtda * (dy * eyr - dy * eyl);
  bz += dtda * (dx * ext - dx * exb);
  o.bz = bz;
  u[BX] = ((I.lv[0][i] - I.lf[0][i]) * o.bxl + (I.lf[0][i + 1] - I.lv[0][i]) * o.bxr) * I.dlf_inv[0][i];
  u[BY] = ((I.lv[1][j] - I.lf[1][j]) * o.byb + (I.lf[1][j + 1] - I.lv[1][j]) * o.byt) * I.dlf_inv[1][j];
  u[BZ] = bz;
  if (I.src) {
    // integrator.pyx:132-170 add_source_terms (bnz_source.cuh)
    double f[3];
    if (I.fdriv) {
      const long long c = (long long)j * I.nx + i;
      f[0] = I.fdriv[c];
      f[1] = I.fdriv[I.sv + c];
      f[2] = I.fdriv[2 * I.sv + c];
    }
    const bool grav = I.grav[0] != 0. || I.grav[1] != 0. || I.grav[2] != 0.;
    srcterm::apply(u, w0[RHO], w0[VX], w0[VY], w0[VZ], I.grav, grav, I.fdriv ? f : nullptr, dt);
  }
  cons2prim(o.w, u, I.gam);
}

// The instance descriptor, copied to shared memory by the first warp so the
// kernels read its fields without global loads.
__device__ __forceinline__ void stage_inst(Inst& sI, const Inst* __restrict__ insts, int q) {
  constexpr int NW = sizeof(Inst) / sizeof(int);
  static_assert(sizeof(Inst) % sizeof(int) == 0, "Inst must be int-aligned");
  const int* src = reinterpret_cast<const int*>(insts + q);
  int* dst = reinterpret_cast<int*>(&sI);
  for (int t = threadIdx.x; t < NW; t += blockDim.x) dst[t] = src[t];
  __syncthreads();
}

// Everything of the predictor after its input is in place: fluxes from the
// cells W and faces F (shared memory, or global memory through the BC map),
// EMFs, the half-step update, the writes of ws / bs.  sF: fluxes and EMFs,
// contiguous (x fluxes, y fluxes, E_c, E_e).
// fail (optional): a flag the block checks at the flux stage's closing barrier;
// when it is set the tile stops there, before writing anything (returns false).
template <int TXM, int TYM, int RS, class Cells, class Faces>
__device__ __forceinline__ bool pred_tile(const Inst& I, const Tile& T, double* sF, const Cells& W, const Faces& F,
                                          double dt, const volatile int* fail = nullptr) {
  using M = Smem<TXM, TYM, 0>;
  double* sFX = sF;
  double* sFY = sFX + NF * M::NFX;
  double* sEC = sFY + NF * M::NFY;
  double* sEE = sEC + M::NEC;
  Layout L;
  L.set_max<TXM, TYM>(T.wx, T.wy);
  unsigned e = 0;
  stage_fluxes<RS>(I, T, L, W, F, sFX, sFY, sEC, e);
  __syncthreads();
  if (fail && *fail) return false;
  stage_emf(L, sFX, sFY, sEC, sEE);
  __syncthreads();
  const int ilast = I.nx - 2, jlast = I.ny - 2;  // last predictor cell (vanleer lims)
  FastDiv dwx;
  dwx.set(T.wx);
  for (int t = threadIdx.x; t < T.wx * T.wy; t += blockDim.x) {
    const int cj = dwx.div(t), ci = t - cj * T.wx;
    const int i = T.x0 + ci, j = T.y0 + cj;
    double wn[NM], un[NM];
    W.load_all(i, j, wn);
    prim2cons(un, wn, I.gam);
    double bxl0 = F.template get<0>(i, j);
    double bxr0 = F.template get<0>(i + 1, j);
    double byb0 = F.template get<1>(i, j);
    double byt0 = F.template get<1>(i, j + 1);
    double bz0 = F.template get<2>(i, j);
    CellOut o;
    stage_cell(I, L, T, ci, cj, un, wn, bxl0, bxr0, byb0, byt0, bz0, sFX, sFY, sEE, dt, o);
    const long long c = (long long)j * I.nx + i;
#pragma unroll
    for (int n = 0; n < NM; ++n) I.ws[n * I.sv + c] = o.w[n];
    I.bs[c] = o.bxl;
    I.bs[I.sv + c] = o.byb;
    I.bs[2 * I.sv + c] = o.bz;
    if (i == ilast) I.bs[c + 1] = o.bxr;
    if (j == jlast) I.bs[I.sv + c + I.nx] = o.byt;
  }
  if (e) atomicOr(I.err, e);
  return true;
}

// a tile whose one-cell ring lies inside the active range needs no ghost mapping
__device__ __forceinline__ bool pred_interior(const Inst& I, const Tile& T) {
  return T.x0 - 1 >= I.ng && T.x0 + T.wx <= I.ng + I.N[0] - 1 && T.y0 - 1 >= I.ng &&
         T.y0 + T.wy <= I.ng + I.N[1] - 1;
}

// Predictor.  STAGED = 1 copies w^n (tile + one ring, BC-mapped) into shared
// memory first; STAGED = 0 reads it from global memory in the flux stage.
template <int TXM, int TYM, int RS, int STAGED>
__global__ void __launch_bounds__(256, 2) k_pred2d(const Inst* __restrict__ insts, const Tile* __restrict__ tiles,
                                                   int parity, int lim) {
  constexpr int RING = STAGED ? 1 : 0;
  extern __shared__ double smem[];
  __shared__ Inst sI;
  const Tile T = tiles[blockIdx.x];
  stage_inst(sI, insts, T.inst);
  const Inst& I = sI;
  const double dtf = I.ds->dt;
  if (!(dtf > 0.)) return;
  const bool interior = pred_interior(I, T);
  // fluxes and EMFs first, then the staged cells
  double* sW = smem + NF * (Smem<TXM, TYM, RING>::NFX + Smem<TXM, TYM, RING>::NFY) + Smem<TXM, TYM, RING>::NEC +
               Smem<TXM, TYM, RING>::NEE;
  Stage S;
  S.x0 = T.x0 - 1;
  S.y0 = T.y0 - 1;
  S.w = T.wx + 2;
  S.h = T.wy + 2;
  const GlobalFaces F{&I, I.b[parity], axis_map(I, 0), axis_map(I, 1), interior};
  if constexpr (STAGED) {
    if (interior) stage_cells<false>(I, I.w[parity], S, sW);
    else stage_cells<true>(I, I.w[parity], S, sW);
    __syncthreads();
    const SmemCells W{sW, S, S.cells()};
    pred_tile<TXM, TYM, RS>(I, T, smem, W, F, 0.5 * dtf);
  } else {
    const GlobalCells W{&I, I.w[parity], axis_map(I, 0), axis_map(I, 1), interior};
    pred_tile<TXM, TYM, RS>(I, T, smem, W, F, 0.5 * dtf);
  }
  (void)lim;
}

__device__ __forceinline__ void copy_tile(const Inst& I, const Tile& T, int parity) {
  const int i2 = I.ng + I.N[0] - 1, j2 = I.ng + I.N[1] - 1;
  const double* w = I.w[parity];
  const double* b = I.b[parity];
  double* w1 = I.w[parity ^ 1];
  double* b1 = I.b[parity ^ 1];
  for (int t = threadIdx.x; t < T.wx * T.wy; t += blockDim.x) {
    const int i = T.x0 + t % T.wx, j = T.y0 + t / T.wx;
    const long long c = (long long)j * I.nx + i;
#pragma unroll
    for (int n = 0; n < NM; ++n) w1[n * I.sv + c] = w[n * I.sv + c];
    for (int n = 0; n < 3; ++n) b1[n * I.sv + c] = b[n * I.sv + c];
    if (i == i2) b1[c + 1] = b[c + 1];
    if (j == j2) b1[I.sv + c + I.nx] = b[I.sv + c + I.nx];
  }
}

// Readers of the corrector's cell-update inputs: w^n and b^n of the cell
// (ghost faces through the BC map) and the half-step state the source terms
// use.  CorrInGlobal reads global memory; CorrInSmem reads w^n / b^n a
// persistent corrector staged by TMA over the tile (edge cells still take
// their faces through the map), and the source-term state from global ws.
struct CorrInGlobal {
  const Inst* I;
  const double* w;
  const double* b;
  const SmemCells* W;
  __device__ __forceinline__ void wn(int i, int j, double* out) const {
    const long long c = (long long)j * I->nx + i;
#pragma unroll
    for (int n = 0; n < NM; ++n) out[n] = w[n * I->sv + c];
  }
  __device__ __forceinline__ double face(int comp, int i, int j, bool edge, const AxisMap& mx,
                                         const AxisMap& my) const {
    if (comp == 0) return load_face<0>(*I, b, i, j, mx, my, !edge);
    if (comp == 1) return load_face<1>(*I, b, i, j, mx, my, !edge);
    return b[2 * I->sv + (long long)j * I->nx + i];
  }
  __device__ __forceinline__ double half(int n, int i, int j) const {
    return W ? W->get(n, i, j) : I->ws[n * I->sv + (long long)j * I->nx + i];
  }
};

struct CorrInSmem {
  const Inst* I;
  const double* b;   // global b^n, for the mapped faces of edge cells
  const double* sw;  // staged w^n (9 fields), layout S
  const double* sb;  // staged b^n (3 faces), layout S
  Stage S;
  __device__ __forceinline__ void wn(int i, int j, double* out) const {
    const int c = S.at(0, i, j);
#pragma unroll
    for (int n = 0; n < NM; ++n) out[n] = sw[n * S.cells() + c];
  }
  __device__ __forceinline__ double face(int comp, int i, int j, bool edge, const AxisMap& mx,
                                         const AxisMap& my) const {
    if (edge && comp == 0) return load_face<0>(*I, b, i, j, mx, my, false);
    if (edge && comp == 1) return load_face<1>(*I, b, i, j, mx, my, false);
    return sb[comp * S.cells() + S.at(0, i, j)];
  }
  __device__ __forceinline__ double half(int n, int i, int j) const {
    return I->ws[n * I->sv + (long long)j * I->nx + i];
  }
};

// The corrector's flux stages: PLM fluxes of every face of the tile and the
// cell-centred EMFs, into sF (x fluxes, y fluxes, E_c, E_e, slopes).  Ends
// with a barrier: the staged half-step cells are no longer needed after it.
template <int TXM, int TYM, int RS, int LIM>
__device__ __forceinline__ void corr_fluxes(const Inst& I, const Tile& T, int cp, const SmemCells& W, double* sF) {
  using M = Smem<TXM, TYM, 2>;
  double* sFX = sF;
  double* sFY = sFX + NF * M::NFX;
  double* sEC = sFY + NF * M::NFY;
  double* sD = sEC + M::NEC + M::NEE;
  Layout L;
  L.set_max<TXM, TYM>(T.wx, T.wy);
  unsigned e = 0;
  stage_fluxes_plm<LIM, RS, (TXM + 2) * (TYM + 2)>(I, T, L, W, I.bs, sFX, sFY, sEC, sD, cp, e);
  if (e) atomicOr(I.err, e);
  __syncthreads();
}

// Corner EMFs, then per cell the full-step update, the writes of w^(n+1) /
// b^(n+1) and the tile's CFL maximum folded into the instance's slot.
template <int TXM, int TYM, class In>
__device__ __forceinline__ void corr_cells(const Inst& I, const Tile& T, int parity, const In& in, double* sF,
                                           double dt, bool emf_done) {
  using M = Smem<TXM, TYM, 2>;
  double* sFX = sF;
  double* sFY = sFX + NF * M::NFX;
  double* sEC = sFY + NF * M::NFY;
  double* sEE = sEC + M::NEC;
  Layout L;
  L.set_max<TXM, TYM>(T.wx, T.wy);
  if (!emf_done) {
    stage_emf(L, sFX, sFY, sEC, sEE);
    __syncthreads();
  }
  unsigned e = 0;
  double* __restrict__ w1 = I.w[parity ^ 1];
  double* __restrict__ b1 = I.b[parity ^ 1];
  const AxisMap mx = axis_map(I, 0), my = axis_map(I, 1);
  const int i2 = I.ng + I.N[0] - 1, j2 = I.ng + I.N[1] - 1;
  double cmax = 0.;
  FastDiv dwx;
  dwx.set(T.wx);
  for (int t = threadIdx.x; t < T.wx * T.wy; t += blockDim.x) {
    const int cj = dwx.div(t), ci = t - cj * T.wx;
    const int i = T.x0 + ci, j = T.y0 + cj;
    const long long c = (long long)j * I.nx + i;
    double wn[NM], un[NM];
    in.wn(i, j, wn);
    prim2cons(un, wn, I.gam);
    // B^n on the cell's faces; the upper boundary face goes through the BC map
    const bool edge = (i == i2) || (j == j2) || (i == I.ng) || (j == I.ng);
    double bxl0 = in.face(0, i, j, edge, mx, my);
    double bxr0 = in.face(0, i + 1, j, edge, mx, my);
    double byb0 = in.face(1, i, j, edge, mx, my);
    double byt0 = in.face(1, i, j + 1, edge, mx, my);
    double bz0 = in.face(2, i, j, edge, mx, my);
    // the corrector's sources use the half-step state ws (vanleer.pyx:143)
    double w0[4] = {0., 0., 0., 0.};
    if (I.src) {
      w0[0] = in.half(RHO, i, j);
      w0[1] = in.half(VX, i, j);
      w0[2] = in.half(VY, i, j);
      w0[3] = in.half(VZ, i, j);
    }
    CellOut o;
    stage_cell(I, L, T, ci, cj, un, w0, bxl0, bxr0, byb0, byt0, bz0, sFX, sFY, sEE, dt, o);
    e |= plain::check_prim(o.w);
#pragma unroll
    for (int n = 0; n < NM; ++n) w1[n * I.sv + c] = o.w[n];
    b1[c] = o.bxl;
    b1[I.sv + c] = o.byb;
    b1[2 * I.sv + c] = o.bz;
    if (i == i2) b1[c + 1] = o.bxr;
    if (j == j2) b1[I.sv + c + I.nx] = o.byt;
    // next step's CFL (new_dt.pyx:55-99) on the new state
    double vf = fms(o.w, I.gam);
    double cx = fabs(o.w[VX]) + vf, cy = fabs(o.w[VY]) + vf;
#if BNZ_FAST_MATH
    double cds = fmax(cx * I.dlf_inv[0][i], cy * I.dlf_inv[1][j]);
#else
    double cds = fmax(fmax(cx / I.dlf[0][i], cy / I.dlf[1][j]), 0. / I.dlf2);
#endif
    if (cds > cmax) cmax = cds;
  }
  // each warp folds its maximum into the slot (positive doubles order as
  // their bit patterns): no block-wide reduction, no barrier
  for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  if ((threadIdx.x & 31) == 0 && cmax > 0.)
    atomicMax(&I.ds->cds_bits[parity ^ 1], (unsigned long long)__double_as_longlong(cmax));
  if (e) atomicOr(I.err, e);
}

// The whole corrector on a tile whose half-step cells are staged in W.
template <int TXM, int TYM, int RS, int LIM>
__device__ __forceinline__ void corr_tile(const Inst& I, const Tile& T, int parity, int cp, const SmemCells& W,
                                          double* sF, double dt) {
  corr_fluxes<TXM, TYM, RS, LIM>(I, T, cp, W, sF);
  const CorrInGlobal in{&I, I.w[parity], I.b[parity], &W};
  corr_cells<TXM, TYM>(I, T, parity, in, sF, dt, false);
}

template <int TXM, int TYM, int RS, int LIM>
__global__ void __launch_bounds__(256, 2) k_corr2d(const Inst* __restrict__ insts, const Tile* __restrict__ tiles,
                                                   int parity, int cp) {
  constexpr int RING = 2;
  extern __shared__ double smem[];
  __shared__ Inst sI;
  const Tile T = tiles[blockIdx.x];
  stage_inst(sI, insts, T.inst);
  const Inst& I = sI;
  const double dt = I.ds->dt;
  if (!(dt > 0.)) {
    // time has reached tmax: carry the state over unchanged
    copy_tile(I, T, parity);
    return;
  }
  // staged cells first, then the fluxes, EMFs and slopes
  double* sW = smem;
  Stage S;
  S.x0 = T.x0 - 2;
  S.y0 = T.y0 - 2;
  S.w = T.wx + 4;
  S.h = T.wy + 4;
  stage_cells<false>(I, I.ws, S, sW);
  __syncthreads();
  SmemCells W{sW, S, S.cells()};
  corr_tile<TXM, TYM, RS, LIM>(I, T, parity, cp, W, smem + Smem<TXM, TYM, RING>::NSW, dt);
}

// ---------------------------------------------------------------------------
// Persistent corrector: a grid of (SMs x resident blocks) takes tiles from a
// work queue (an atomic counter the dt kernel resets every step).  The staged
// input (ws on the tile and two rings, 9 fields) of the NEXT tile is loaded by
// TMA into the second of two shared-memory buffers while the current tile is
// computed.  The TMA box starts at an even column (16-byte rule for FP64) and
// is TmaBox::W cells wide; rows or columns past the array read as zeros and
// are never used.  Instances whose rows are not a multiple of 16 bytes
// (odd Ntot_x) have no tensor map: their tiles stage with plain loads.
// ---------------------------------------------------------------------------

template <int TXM, int TYM>
struct TmaBox {
  static constexpr int W = (TXM + 5 + 1) & ~1;  // TX+4 cells from an even column at or before x0-2
  static constexpr int H = TYM + 4;
  static constexpr int CELLS = W * H;
  static constexpr unsigned BYTES = NM * CELLS * sizeof(double);
  static constexpr int BUF = (NM * CELLS + 15) / 16 * 16;  // doubles per buffer, 128-byte multiple
  // the cell update's w^n and b^n on the tile (faces up to x0+TX, y0+TY),
  // loaded into the same buffer once the flux stages are done with it
  static constexpr int CW = (TXM + 3) & ~1;  // TX+1 positions from an even column at or before x0
  static constexpr int CH = TYM + 1;
  static constexpr int CCELLS = CW * CH;
  static constexpr int COFF = (NM * CCELLS + 15) / 16 * 16;  // b^n box, 128-byte aligned
  static constexpr unsigned CBYTES = (NM + 3) * CCELLS * sizeof(double);
  static_assert(COFF + 3 * CCELLS <= BUF, "the cell-update boxes must fit one staging buffer");
  static constexpr size_t smem_bytes = 128 +  // room to align the buffers
      sizeof(double) * (2 * (size_t)BUF + (size_t)NF * (Smem<TXM, TYM, 2>::NFX + Smem<TXM, TYM, 2>::NFY) +
                        Smem<TXM, TYM, 2>::NEC + Smem<TXM, TYM, 2>::NEE + Smem<TXM, TYM, 2>::NSD);
};

namespace tma {
__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_bar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ void arrive_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool try_wait(unsigned long long* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(phase)
      : "memory");
  return ok != 0u;
}
// bounded wait: false after about a second without the phase completing
__device__ __forceinline__ bool wait(unsigned long long* bar, unsigned phase) {
  const long long t0 = clock64();
  while (!try_wait(bar, phase))
    if (clock64() - t0 > (1LL << 31)) return false;
  return true;
}
__device__ __forceinline__ void load_3d(void* dst, unsigned long long* bar, const void* map, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(saddr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(saddr(bar))
      : "memory");
}
// the box of a tensor map at (x, y, z) into L2, no shared memory involved
__device__ __forceinline__ void prefetch_l2_3d(const void* map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global [%0, {%1, %2, %3}];" ::"l"(map), "r"(x), "r"(y), "r"(z)
               : "memory");
}
__device__ __forceinline__ void prefetch_map(const void* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}
}  // namespace tma

// Issued by one thread for the tile that will use buffer dst / bar: its
// staged input by TMA, or (no tensor map) a plain arrival, so that the
// barrier's phase completes either way.
template <int TXM, int TYM>
__device__ __forceinline__ void issue_ws(const Tile& T, const unsigned char* maps, double* dst,
                                         unsigned long long* bar, int withhold) {
  if (T.tma) {
    const void* map = maps + (size_t)T.inst * 6 * 128;
    tma::fence_async_shared();
    tma::arrive_expect(bar, TmaBox<TXM, TYM>::BYTES);
    if (!withhold) tma::load_3d(dst, bar, map, (T.x0 - 2) & ~1, T.y0 - 2, 0);
  } else {
    tma::arrive(bar);
  }
}

// Issued with the staged input of the next tile: its flux stage's normal
// faces of bs (map 5: bx, by over the faces the flux stage reads) and its
// cell update's w^n / b^n, brought into L2 a tile ahead.
template <int TXM, int TYM>
__device__ __forceinline__ void prefetch_next(const Tile& T, const unsigned char* maps, int parity) {
  if (!T.tma) return;
  const unsigned char* m = maps + (size_t)T.inst * 6 * 128;
  tma::prefetch_l2_3d(m + 5 * 128, (T.x0 - 1) & ~1, T.y0 - 1, 0);
  tma::prefetch_l2_3d(m + (1 + parity) * 128, T.x0 & ~1, T.y0, 0);
  tma::prefetch_l2_3d(m + (3 + parity) * 128, T.x0 & ~1, T.y0, 0);
}

// The cell update's w^n (cells of the tile) and b^n (faces up to x0+wx,
// y0+wy) with plain loads into the layout S of the cell-update TMA boxes:
// the staging of tiles that have no TMA load.  Faces on the domain boundary
// are read through the BC map later, as with TMA.
__device__ __forceinline__ void stage_corr_inputs(const Inst& I, const Tile& T, int parity, const Stage& S, int boff,
                                                  double* sW) {
  const double* __restrict__ w = I.w[parity];
  const double* __restrict__ b = I.b[parity];
  const int rw = T.wx + 1, n = rw * (T.wy + 1);
  FastDiv dw;
  dw.set(rw);
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int cj = dw.div(t), ci = t - cj * rw;
    const int i = T.x0 + ci, j = T.y0 + cj;
    const long long c = (long long)j * I.nx + i;
    const int d = S.at(0, i, j);
    if (ci < T.wx && cj < T.wy) {
#pragma unroll
      for (int q = 0; q < NM; ++q) sW[q * S.cells() + d] = w[q * I.sv + c];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) sW[boff + q * S.cells() + d] = b[q * I.sv + c];
  }
}

// Issued by one thread once the tile's flux stages are done with buffer dst:
// w^n and b^n of the tile for the cell update (maps 1 + parity and 3 + parity
// of the instance), or a plain arrival.
template <int TXM, int TYM>
__device__ __forceinline__ void issue_wn(const Tile& T, const unsigned char* maps, int parity, double* dst,
                                         unsigned long long* bar, int withhold) {
  using B = TmaBox<TXM, TYM>;
  if (T.tma) {
    const unsigned char* m = maps + (size_t)T.inst * 6 * 128;
    const int x = T.x0 & ~1, y = T.y0;
    tma::fence_async_shared();
    tma::arrive_expect(bar, B::CBYTES);
    if (!withhold) {
      tma::load_3d(dst, bar, m + (1 + parity) * 128, x, y, 0);
      tma::load_3d(dst + B::COFF, bar, m + (3 + parity) * 128, x, y, 0);
    }
  } else {
    tma::arrive(bar);
  }
}

// Iteration k of a block uses buffer, instance slot and tile slot k & 1.
// Each buffer use completes two phases of that buffer's barrier: the staged
// half-step input (parity 0), then the cell update's w^n / b^n (parity 1),
// loaded once the flux stages are done.  The next tile's instance record is
// copied at the end of the current tile, so the barrier that ends a tile also
// publishes the next one: every thread then waits on the TMA barrier itself,
// and a wait that ran out is acted on at the flux stage's closing barrier,
// before the tile writes anything.
// withhold (a test switch, 0 in every normal call): the TMA loads are armed on
// their barriers but not issued, so that the bounded waits run out.
template <int TXM, int TYM, int RS, int LIM>
__global__ void __launch_bounds__(256, 2) k_corr2d_pq(const Inst* __restrict__ insts, const Tile* __restrict__ tiles,
                                                      int ntiles, int parity, int cp,
                                                      const unsigned char* __restrict__ maps,
                                                      unsigned* __restrict__ queue, int withhold) {
  using B = TmaBox<TXM, TYM>;
  using M = Smem<TXM, TYM, 2>;
  extern __shared__ __align__(128) double smem_raw[];
  __shared__ Inst sI[2];
  __shared__ Tile sT[2];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int s_tile[2], s_fail;  // tile of iteration k in s_tile[k & 1]
  // TMA destinations start on 128-byte boundaries (the launch adds 128 bytes)
  double* smem = smem_raw + ((128u - (tma::saddr(smem_raw) & 127u)) & 127u) / sizeof(double);
  // two staging buffers of B::BUF doubles, then the fluxes, EMFs and slopes
  if (threadIdx.x == 0) {
    tma::bar_init(&bar[0], 1);
    tma::bar_init(&bar[1], 1);
    tma::fence_bar_init();
    s_fail = 0;
    const int t0 = (int)atomicAdd(queue, 1u);
    s_tile[0] = t0;
    if (t0 < ntiles) {
      const Tile T0 = tiles[t0];
      sT[0] = T0;
      if (T0.tma) tma::prefetch_map(maps + (size_t)T0.inst * 6 * 128);
      issue_ws<TXM, TYM>(T0, maps, smem, &bar[0], withhold);
      prefetch_next<TXM, TYM>(T0, maps, parity);
    }
  }
  __syncthreads();
  if (s_tile[0] < ntiles) stage_inst(sI[0], insts, sT[0].inst);  // ends with a barrier
  for (int k = 0;; ++k) {
    // written by thread 0 before the last barrier; the slot it writes next
    // was last read before an earlier barrier
    const int t = s_tile[k & 1];
    if (t >= ntiles) break;
    const int buf = k & 1;
    double* sW = smem + buf * B::BUF;
    if (threadIdx.x == 0) {
      const int tn = (int)atomicAdd(queue, 1u);
      s_tile[buf ^ 1] = tn;
      // the other buffer is free: its tile finished before the last barrier
      if (tn < ntiles) {
        const Tile TN = tiles[tn];
        issue_ws<TXM, TYM>(TN, maps, smem + (buf ^ 1) * B::BUF, &bar[buf ^ 1], withhold);
        prefetch_next<TXM, TYM>(TN, maps, parity);
      }
    }
    const Tile& T = sT[buf];
    const Inst& I = sI[buf];
    // this tile's staged input, each thread for itself (bounded)
    if (!tma::wait(&bar[buf], 0u)) s_fail = 1;
    const double dt = I.ds->dt;
    bool alive = true;
    if (!(dt > 0.)) {
      copy_tile(I, T, parity);  // time has reached tmax: carry the state over (no staged data used)
      // every thread has passed its parity-0 wait before phase 1 can complete
      __syncthreads();
    } else {
      // the TMA box's layout in both cases (compile-time sizes)
      Stage S;
      S.x0 = (T.x0 - 2) & ~1;
      S.y0 = T.y0 - 2;
      S.w = B::W;
      S.h = B::H;
      if (!T.tma) {
        Stage R;
        R.x0 = T.x0 - 2;
        R.y0 = T.y0 - 2;
        R.w = T.wx + 4;
        R.h = T.wy + 4;
        stage_cells_into(I, I.ws, R, S, sW);
        __syncthreads();
      }
      const SmemCells W{sW, S, S.cells()};
      corr_fluxes<TXM, TYM, RS, LIM>(I, T, cp, W, smem + 2 * B::BUF);  // ends with a barrier
      alive = !s_fail;
    }
    if (alive) {
      // the flux stages are done with the buffer: the cell update's inputs
      if (threadIdx.x == 0) {
        if (T.tma && dt > 0.) issue_wn<TXM, TYM>(T, maps, parity, sW, &bar[buf], withhold);
        else tma::arrive(&bar[buf]);
      }
      if (dt > 0.) {
        Layout L;
        L.set_max<TXM, TYM>(T.wx, T.wy);
        double* sF = smem + 2 * B::BUF;
        stage_emf(L, sF, sF + NF * M::NFX, sF + NF * (M::NFX + M::NFY), sF + NF * (M::NFX + M::NFY) + M::NEC);
      }
      // one thread waits (bounded) and tells the block; then every thread
      // observes the completed phase itself
      if (threadIdx.x == 0 && !tma::wait(&bar[buf], 1u)) s_fail = 1;
      __syncthreads();
      alive = !s_fail;
    }
    if (!alive) {
      // flag it, give the next tile's load (if any) a bounded wait, and leave
      if (threadIdx.x == 0) {
        atomicOr(I.err, (unsigned)ERR_TIMEOUT);
        if (s_tile[buf ^ 1] < ntiles) tma::wait(&bar[buf ^ 1], 0u);
      }
      return;
    }
    tma::wait(&bar[buf], 1u);
    if (dt > 0.) {
      // the TMA boxes' layout in both cases (compile-time sizes)
      Stage S;
      S.x0 = T.x0 & ~1;
      S.y0 = T.y0;
      S.w = B::CW;
      S.h = B::CH;
      if (!T.tma) {
        stage_corr_inputs(I, T, parity, S, B::COFF, sW);
        __syncthreads();
      }
      const CorrInSmem in{&I, I.b[parity], sW, sW + B::COFF, S};
      corr_cells<TXM, TYM>(I, T, parity, in, smem + 2 * B::BUF, dt, true);
    }
    // the next tile's records into the other slots (last used by the tile
    // before this one), published by the barrier that ends this tile
    const int tn = s_tile[buf ^ 1];
    if (tn < ntiles) {
      if (threadIdx.x == 0) sT[buf ^ 1] = tiles[tn];
      const int* src = reinterpret_cast<const int*>(insts + tiles[tn].inst);
      int* dst = reinterpret_cast<int*>(&sI[buf ^ 1]);
      for (int q = threadIdx.x; q < (int)(sizeof(Inst) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();  // the tile's buffer and slots are free; the next tile's are set
  }
}

// Persistent predictor: the same work queue and double buffering as the
// persistent corrector.  Its tiles cover the predictor range (cells 1 ..
// Ntot-2) in plain tx x ty steps, so none is larger than tx x ty.  Interior
// tiles (full tiles whose one-cell ring lies inside the active range, so no
// ghost is read) get w^n (9 fields) and b^n (3 faces) on the tile and its ring
// by two TMA loads into one buffer; the other tiles stage them with plain
// loads through the BC map into the same layout.  The boxes start at an even
// column and are TmaBoxP::W cells wide.
template <int TX, int TY>
struct TmaBoxP {
  static constexpr int W = (TX + 4) & ~1;  // TX+2 cells from an even column at or before x0-1
  static constexpr int H = TY + 2;
  static constexpr int CELLS = W * H;
  static constexpr unsigned WBYTES = NM * CELLS * sizeof(double);
  static constexpr unsigned BYTES = (NM + 3) * CELLS * sizeof(double);
  static constexpr int BUF = ((NM + 3) * CELLS + 15) / 16 * 16;
  static_assert(WBYTES % 128 == 0, "the face box must start on a 128-byte boundary");
  using M = Smem<TX, TY, 0>;
  static constexpr size_t smem_bytes =
      128 + sizeof(double) * (2 * (size_t)BUF + (size_t)NF * (M::NFX + M::NFY) + M::NEC + M::NEE);
};

// maps: 4 per instance, w[0], w[1], b[0], b[1]
// T.tma: 1 = staged by TMA; 2 = an edge tile of an instance with maps, whose
// own box of w^n / b^n is brought into L2 (its reads go through the BC map);
// 0 = neither.
template <int TX, int TY>
__device__ __forceinline__ void issue_wb(const Tile& T, const unsigned char* maps, int parity, double* dst,
                                         unsigned long long* bar, int withhold) {
  if (T.tma == 2) {
    const unsigned char* m = maps + (size_t)T.inst * 4 * 128;
    tma::prefetch_l2_3d(m + parity * 128, (T.x0 - 1) & ~1, T.y0 - 1, 0);
    tma::prefetch_l2_3d(m + (2 + parity) * 128, (T.x0 - 1) & ~1, T.y0 - 1, 0);
  }
  if (T.tma == 1) {
    const unsigned char* m = maps + (size_t)T.inst * 4 * 128;
    const int x = (T.x0 - 1) & ~1, y = T.y0 - 1;
    tma::fence_async_shared();
    tma::arrive_expect(bar, TmaBoxP<TX, TY>::BYTES);
    if (!withhold) {
      tma::load_3d(dst, bar, m + parity * 128, x, y, 0);
      tma::load_3d(dst + NM * TmaBoxP<TX, TY>::CELLS, bar, m + (2 + parity) * 128, x, y, 0);
    }
  } else {
    tma::arrive(bar);
  }
}

// The predictor's inputs of tile T (cells and faces on the tile and its ring,
// ghost positions through the BC map) into the layout S of a TMA box: the
// staging of tiles that have no TMA load.
__device__ __forceinline__ void stage_pred_mapped(const Inst& I, const Tile& T, int parity, const Stage& S,
                                                  double* sW, bool interior) {
  const double* __restrict__ w = I.w[parity];
  const double* __restrict__ b = I.b[parity];
  const AxisMap mx = axis_map(I, 0), my = axis_map(I, 1);
  const int rw = T.wx + 2, n = rw * (T.wy + 2);
  FastDiv dw;
  dw.set(rw);
  double* sB = sW + NM * S.cells();
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int cj = dw.div(t), ci = t - cj * rw;
    const int i = T.x0 - 1 + ci, j = T.y0 - 1 + cj;
    const int d = S.at(0, i, j);
    double v[NM];
    load_prim_all(I, w, i, j, mx, my, interior, v);
#pragma unroll
    for (int q = 0; q < NM; ++q) sW[q * S.cells() + d] = v[q];
    sB[d] = load_face<0>(I, b, i, j, mx, my, interior);
    sB[S.cells() + d] = load_face<1>(I, b, i, j, mx, my, interior);
    sB[2 * S.cells() + d] = load_face<2>(I, b, i, j, mx, my, interior);
  }
}

// Iteration k uses buffer, instance slot and tile slot k & 1; each buffer use
// completes one phase of its barrier.  As in the persistent corrector, the
// next tile's records are copied at the end of the current tile and every
// thread waits on the TMA barrier itself; a wait that ran out is acted on at
// the flux stage's closing barrier (or at the top of the next tile).
template <int TX, int TY, int RS>
__global__ void __launch_bounds__(256, 2) k_pred2d_pq(const Inst* __restrict__ insts, const Tile* __restrict__ tiles,
                                                      int ntiles, int parity, const unsigned char* __restrict__ maps,
                                                      unsigned* __restrict__ queue, int withhold) {
  using B = TmaBoxP<TX, TY>;
  extern __shared__ __align__(128) double smem_raw[];
  __shared__ Inst sI[2];
  __shared__ Tile sT[2];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int s_tile[2];  // tile of iteration k in s_tile[k & 1]
  __shared__ volatile int s_fail;
  double* smem = smem_raw + ((128u - (tma::saddr(smem_raw) & 127u)) & 127u) / sizeof(double);
  // two staging buffers of B::BUF doubles, then the fluxes and EMFs
  if (threadIdx.x == 0) {
    tma::bar_init(&bar[0], 1);
    tma::bar_init(&bar[1], 1);
    tma::fence_bar_init();
    s_fail = 0;
    const int t0 = (int)atomicAdd(queue, 1u);
    s_tile[0] = t0;
    if (t0 < ntiles) {
      const Tile T0 = tiles[t0];
      sT[0] = T0;
      if (T0.tma == 1) {
        tma::prefetch_map(maps + ((size_t)T0.inst * 4 + parity) * 128);
        tma::prefetch_map(maps + ((size_t)T0.inst * 4 + 2 + parity) * 128);
      }
      issue_wb<TX, TY>(T0, maps, parity, smem, &bar[0], withhold);
    }
  }
  __syncthreads();
  if (s_tile[0] < ntiles) stage_inst(sI[0], insts, sT[0].inst);  // ends with a barrier
  for (int k = 0;; ++k) {
    const int t = s_tile[k & 1];
    const int buf = k & 1;
    const Inst& I = sI[buf];
    if (s_fail) {
      // a load did not complete: flag it, give the load in flight (if any) a
      // bounded wait, and leave
      if (threadIdx.x == 0) {
        atomicOr(I.err, (unsigned)ERR_TIMEOUT);
        if (t < ntiles) tma::wait(&bar[buf], (unsigned)(k >> 1) & 1u);
      }
      return;
    }
    if (t >= ntiles) break;
    if (threadIdx.x == 0) {
      const int tn = (int)atomicAdd(queue, 1u);
      s_tile[buf ^ 1] = tn;
      if (tn < ntiles) issue_wb<TX, TY>(tiles[tn], maps, parity, smem + (buf ^ 1) * B::BUF, &bar[buf ^ 1], withhold);
    }
    const Tile& T = sT[buf];
    // this tile's input, each thread for itself (bounded)
    if (!tma::wait(&bar[buf], (unsigned)(k >> 1) & 1u)) s_fail = 1;
    const double dtf = I.ds->dt;
    if (dtf > 0.) {
      // the TMA box's layout in both cases (compile-time sizes)
      Stage S;
      S.x0 = (T.x0 - 1) & ~1;
      S.y0 = T.y0 - 1;
      S.w = B::W;
      S.h = B::H;
      double* sW = smem + buf * B::BUF;
      if (T.tma != 1) {
        stage_pred_mapped(I, T, parity, S, sW, pred_interior(I, T));
        __syncthreads();
      }
      const SmemCells W{sW, S, S.cells()};
      const SmemFaces F{sW + NM * B::CELLS, S};
      if (!pred_tile<TX, TY, RS>(I, T, smem + 2 * B::BUF, W, F, 0.5 * dtf, &s_fail)) {
        if (threadIdx.x == 0) {
          atomicOr(I.err, (unsigned)ERR_TIMEOUT);
          if (s_tile[buf ^ 1] < ntiles) tma::wait(&bar[buf ^ 1], (unsigned)((k + 1) >> 1) & 1u);
        }
        return;
      }
    } else {
      // no work on this tile (time at tmax): thread 0's s_tile write above
      // must still be visible before the next tile's records are read below
      __syncthreads();
    }
    // the next tile's records into the other slots, published by the barrier
    // that ends this tile
    const int tn = s_tile[buf ^ 1];
    if (tn < ntiles) {
      if (threadIdx.x == 0) sT[buf ^ 1] = tiles[tn];
      const int* src = reinterpret_cast<const int*>(insts + tiles[tn].inst);
      int* dst = reinterpret_cast<int*>(&sI[buf ^ 1]);
      for (int q = threadIdx.x; q < (int)(sizeof(Inst) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();  // the tile's buffer and slots are free; the next tile's are set
  }
}

// Per-instance dt for the step of parity p (new_dt.pyx:117, vanleer.pyx:95-96):
// FDT_CFL  cour / max of slot p, clipped to tmax;
// FDT_FIXED dt_fixed (the FIXDT build), clipped to tmax;
// FDT_EXPLICIT keeps the dt the host wrote (bnz_vl2_step).
// Clears the slot the corrector fills for the next step (or carries the slot
// over when the step does not advance), and the persistent corrector's
// work-queue counter.
// (IT: the instance record of the 2D or the 3D kernels; only its ds is read)
template <class IT>
__global__ void k_dt_batch(const IT* __restrict__ insts, int n, int parity, double cour, int mode, double dt_fixed,
                           unsigned* queue) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q == 0 && queue) queue[0] = queue[1] = 0u;  // the persistent kernels' tile counters
  if (q >= n) return;
  DtState* ds = insts[q].ds;
  if (mode != FDT_EXPLICIT) {
    double dt;
    if (mode == FDT_FIXED) {
      dt = dt_fixed;
    } else {
      double m = __longlong_as_double((long long)ds->cds_bits[parity]);
      dt = cour / m;
      if (ds->time + dt > ds->tmax) dt = ds->tmax - ds->time;
    }
    if (ds->time >= ds->tmax) dt = 0.;
    ds->dt = dt;
  }
  // a step that does not advance (time at tmax) leaves the state, and so its
  // CFL maximum, unchanged: the slot is carried over instead of refilled
  ds->cds_bits[parity ^ 1] = ds->dt > 0. ? 0ULL : ds->cds_bits[parity];
}

template <class IT>
__global__ void k_time_batch(const IT* __restrict__ insts, int n) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  DtState* ds = insts[q].ds;
  if (ds->dt > 0.) {
    ds->time += ds->dt;
    ds->step += 1;
  }
}

// CFL max of the current state into slot `parity` (new_dt.pyx:18-135): the
// first step of a run, or after the state was replaced.
__global__ void k_cds_batch(const Inst* __restrict__ insts, const Tile* __restrict__ tiles, int parity) {
  __shared__ double red[8];
  const Tile T = tiles[blockIdx.x];
  const Inst& I = insts[T.inst];
  const double* w = I.w[parity];
  double cmax = 0.;
  for (int t = threadIdx.x; t < T.wx * T.wy; t += blockDim.x) {
    const int i = T.x0 + t % T.wx, j = T.y0 + t / T.wx;
    const long long c = (long long)j * I.nx + i;
    double ww[NM];
#pragma unroll
    for (int n = 0; n < NM; ++n) ww[n] = w[n * I.sv + c];
    double vf = fms(ww, I.gam);
    double cx = fabs(ww[VX]) + vf, cy = fabs(ww[VY]) + vf;
    double cds = fmax(fmax(cx / I.dlf[0][i], cy / I.dlf[1][j]), 0. / I.dlf2);
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

}  // namespace fused
