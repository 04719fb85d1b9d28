// bnz_adjoint.cuh -- discrete adjoint (reverse mode) of one 2D VL2 step of
// the fused path: given the cotangent of the step's output state, the
// cotangent of its input state.  Hand-written; the reference has no adjoint.
//
// The forward step (bnz_fused.cuh) is a function of the state's SOURCE values
// (active cells, the faces the CT update owns): every read outside them goes
// through the boundary-condition index maps, and the stored output is what the
// ghost fill would leave.  The reverse step mirrors that:
//   fold     the output cotangent through the index maps onto the sources;
//   stage 1  corrector  (order 1, dt,   active cells)   -> cotangents of the
//            predictor output (ws, bs) and of the reads of w^n, b^n;
//   stage 0  predictor  (order 0, dt/2, cells 1..Ntot-2) -> reads of w^n, b^n;
//   fold     the accumulated read cotangents ("virtual" positions, ghosts
//            included) onto the sources of w^n, b^n.
// Each stage is four gathers with no atomics: per cell the EOS VJP, per corner
// the EMF cotangent, per face the flux cotangent and the Riemann + PLM VJP
// (bnz_adjoint_math.h), per cell the sum over the faces that read it.  The
// forward values come from the recorded states (w^n, b^n, ws, bs, w^(n+1)).
// Included inside the per-floating-point-mode namespace.
#pragma once

#ifndef BNZ_ADJ_FACE_MINB
#define BNZ_ADJ_FACE_MINB 1  // blocks of 128 per SM the face kernel is compiled for (register budget)
#endif

namespace adjk {

using namespace fused;  // Inst, AxisMap, map_cell, map_face

struct Box {
  int ia, ib, ja, jb;  // inclusive cell range of the stage's update
};

struct StageArgs {
  int order;
  int charact;          // order 1 with charact_proj: projected slopes, the cells' normal B read too
  double dt;
  Box R;
  const double* Wout;   // the stage's output prim (9)
  const double* Gw;     // its cotangent (9)
  const double* Gb;     // cotangent of the output faces (3)
  const double* Wsrc;   // cells the fluxes read (order 1: ws; order 0: w^n, mapped)
  const double* Bsrc;   // faces the fluxes read (order 1: bs; order 0: b^n, mapped)
  const double* Wn;     // w^n (the u^n of the update is prim2cons of it)
  double* Vw;           // += cotangent of the reads of w^n (virtual positions)
  double* Vb;           // += cotangent of the reads of b^n
  double* Wsrc_b;       // order 1: = cotangent of ws (set); order 0: Vw
  double* Bsrc_b;       // order 1: = cotangent of bs (set); order 0: Vb
  double* Ub;           // scratch: cotangent of the updated conserved state (9)
  double* Eb;           // scratch: cotangent of the corner EMF
  double* Q;            // scratch: per-face Riemann/PLM cotangents, [ax][slot 0..3][var][face]
};

__device__ __forceinline__ long long cidx(const Inst& I, int i, int j) { return (long long)j * I.nx + i; }

__device__ __forceinline__ bool in(const Box& R, int i, int j) {
  return i >= R.ia && i <= R.ib && j >= R.ja && j <= R.jb;
}

// prim at (i, j): mapped read (order 0, w^n) or direct (order 1, ws)
__device__ __forceinline__ void read_cell(const Inst& I, const double* w, int i, int j, bool map, double* out) {
  bool fx = false, fy = false;
  int si = i, sj = j;
  if (map) {
    si = map_cell(i, axis_map(I, 0), fx);
    sj = map_cell(j, axis_map(I, 1), fy);
  }
  const long long c = cidx(I, si, sj);
#pragma unroll
  for (int n = 0; n < NM; ++n) {
    double v = w[n * I.sv + c];
    if ((fx && (n == VX || n == BX)) || (fy && (n == VY || n == BY))) v = -v;
    out[n] = v;
  }
}

template <int COMP>
__device__ __forceinline__ double read_face(const Inst& I, const double* b, int i, int j, bool map) {
  if (!map) return b[COMP * I.sv + cidx(I, i, j)];
  return load_face<COMP>(I, b, i, j, axis_map(I, 0), axis_map(I, 1), false);
}

// u[BX] = cl(i) bx(i) + cr(i) bx(i+1) (ct.pyx:96-123 on a uniform or stretched axis)
__device__ __forceinline__ double cl(const Inst& I, int ax, int i) {
  return (I.lv[ax][i] - I.lf[ax][i]) * I.dlf_inv[ax][i];
}
__device__ __forceinline__ double cr(const Inst& I, int ax, int i) {
  return (I.lf[ax][i + 1] - I.lv[ax][i]) * I.dlf_inv[ax][i];
}

// Cotangent of the output face field including the cell-centred B it feeds
// (x face (i, j) for AX = 0 with j in the output rows; y face for AX = 1).
template <int AX>
__device__ __forceinline__ double face_total(const Inst& I, const StageArgs& a, int i, int j) {
  const Box& R = a.R;
  double g = a.Gb[AX * I.sv + cidx(I, i, j)];
  if (AX == 0) {
    if (i - 1 >= R.ia) g += cr(I, 0, i - 1) * a.Ub[BX * I.sv + cidx(I, i - 1, j)];
    if (i <= R.ib) g += cl(I, 0, i) * a.Ub[BX * I.sv + cidx(I, i, j)];
  } else {
    if (j - 1 >= R.ja) g += cr(I, 1, j - 1) * a.Ub[BY * I.sv + cidx(I, i, j - 1)];
    if (j <= R.jb) g += cl(I, 1, j) * a.Ub[BY * I.sv + cidx(I, i, j)];
  }
  return g;
}

__device__ __forceinline__ double bz_total(const Inst& I, const StageArgs& a, int i, int j) {
  const long long c = cidx(I, i, j);
  return a.Gb[2 * I.sv + c] + a.Ub[BZ * I.sv + c];
}

// Constant gravity, added after a stage's update (bnz_source.cuh
// srcterm::apply): u[M] += dt rho g, u[EN] += dt rho v.g, with rho and v of
// the stage input.  Its VJP adds ubar's share onto that input's prim.
__device__ __forceinline__ bool grav_on(const Inst& I) {
  return I.grav[0] != 0. || I.grav[1] != 0. || I.grav[2] != 0.;
}
__device__ __forceinline__ void grav_vjp(const Inst& I, double dt, const double* ub, double rho, double vx, double vy,
                                         double vz, double* wb) {
  const double* g = I.grav;
  const double e = dt * ub[EN];
  wb[RHO] += dt * (g[0] * ub[MX] + g[1] * ub[MY] + g[2] * ub[MZ]) + e * (vx * g[0] + vy * g[1] + vz * g[2]);
  wb[VX] += e * rho * g[0];
  wb[VY] += e * rho * g[1];
  wb[VZ] += e * rho * g[2];
}

// --- S1: per updated cell, ubar = VJP of cons2prim at the output; the
// prim2cons of w^n that forms u^n gets ubar's hydro part; the predictor's
// gravity term (stage input w^n) too --------------------------------------
__device__ __forceinline__ void cells_body(const Inst& I, const StageArgs& a, int i, int j, const double* g) {
  const long long c = cidx(I, i, j);
  double wo[NM], ub[NM];
#pragma unroll
  for (int v = 0; v < NM; ++v) {
    wo[v] = a.Wout[v * I.sv + c];
    ub[v] = 0.;
  }
  adj::vjp_cons2prim(wo, g, I.gam, ub);
#pragma unroll
  for (int v = 0; v < NM; ++v) a.Ub[v * I.sv + c] = ub[v];
  // u^n = prim2cons(w^n); its B entries are replaced by the face averages
  double wn[NM], wb[NM];
  read_cell(I, a.Wn, i, j, a.order == 0, wn);
  ub[BX] = ub[BY] = ub[BZ] = 0.;
#pragma unroll
  for (int v = 0; v < NM; ++v) wb[v] = 0.;
  adj::vjp_prim2cons(wn, ub, I.gam, wb);
  if (a.order == 0 && grav_on(I)) grav_vjp(I, a.dt, ub, wn[RHO], wn[VX], wn[VY], wn[VZ], wb);
#pragma unroll
  for (int v = 0; v < NM; ++v) a.Vw[v * I.sv + c] += wb[v];
}

__global__ void k_cells(const Inst I, const StageArgs a) {
  const Box R = a.R;
  const int w = R.ib - R.ia + 1;
  const long long n = (long long)w * (R.jb - R.ja + 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = R.ia + (int)(t % w), j = R.ja + (int)(t / w);
    const long long c = cidx(I, i, j);
    double g[NM];
#pragma unroll
    for (int v = 0; v < NM; ++v) g[v] = a.Gw[v * I.sv + c];
    cells_body(I, a, i, j, g);
  }
}

// --- S2: per corner, the cotangent of the corner EMF (ct.pyx:15-91) ------
__global__ void k_corners(const Inst I, const StageArgs a) {
  const Box R = a.R;
  const int w = R.ib - R.ia + 2;
  const long long n = (long long)w * (R.jb - R.ja + 2);
  const double dz = I.dlf2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = R.ia + (int)(t % w), j = R.ja + (int)(t / w);
    double e = 0.;
    // x faces (i, j) and (i, j-1): bx -= dt/(dy dz) (dz E(i,j+1) - dz E(i,j))
    if (j <= R.jb) e += face_total<0>(I, a, i, j) * (a.dt / (I.dlf[1][j] * dz)) * dz;
    if (j - 1 >= R.ja) e -= face_total<0>(I, a, i, j - 1) * (a.dt / (I.dlf[1][j - 1] * dz)) * dz;
    // y faces (i, j) and (i-1, j): by += dt/(dx dz) (dz E(i+1,j) - dz E(i,j))
    if (i <= R.ib) e -= face_total<1>(I, a, i, j) * (a.dt / (I.dlf[0][i] * dz)) * dz;
    if (i - 1 >= R.ia) e += face_total<1>(I, a, i - 1, j) * (a.dt / (I.dlf[0][i - 1] * dz)) * dz;
    a.Eb[cidx(I, i, j)] = e;
  }
}

__device__ __forceinline__ double corner_b(const Inst& I, const StageArgs& a, int i, int j) {
  const Box& R = a.R;
  if (i < R.ia || i > R.ib + 1 || j < R.ja || j > R.jb + 1) return 0.;
  return a.Eb[cidx(I, i, j)];
}

// --- S3: per face, the flux cotangent, the Riemann VJP and the PLM VJP ----
// The PLM stencil is not kept live across the Riemann VJP: the face states are
// built, the stencil dropped, and the four cells reloaded (L1) for the PLM VJP.
template <int AX, int ORDER>
__device__ __forceinline__ double plm_cell(const Inst& I, const double* W, int i, int j, int q, int gv) {
  const int ci = AX == 0 ? i - 2 + q : i, cj = AX == 0 ? j : j - 2 + q;
  return W[gv * I.sv + cidx(I, ci, cj)];
}

// x faces: i in [ia, ib+1], rows [ja-1, jb+1]; y faces: rows [ja, jb+1], columns [ia-1, ib+1]
template <int AX>
__device__ __forceinline__ void face_range(const Box& R, int& fi0, int& fj0, int& w, long long& n) {
  fi0 = AX == 0 ? R.ia : R.ia - 1;
  fj0 = AX == 0 ? R.ja - 1 : R.ja;
  w = R.ib + 1 - fi0 + 1;
  n = (long long)w * (R.jb + 1 - fj0 + 1);
}

template <int AX, int ORDER, int RS, bool CHAR>
__device__ __forceinline__ void face_vjp(const Inst& I, const StageArgs& a, int lim, long long t) {
  const Box R = a.R;
  int fi0, fj0, w;
  long long n;
  face_range<AX>(R, fi0, fj0, w, n);
  const double dz = I.dlf2;
  {
    const int i = fi0 + (int)(t % w), j = fj0 + (int)(t / w);
    const long long f = cidx(I, i, j);
    // the two cells this face separates: (il, jl) and (i, j)
    const int il = AX == 0 ? i - 1 : i, jl = AX == 0 ? j : j - 1;
    const bool inL = in(R, il, jl), inR = in(R, i, j);
    // flux cotangent, local frame of the sweep (godunov.pyx:297-324 permutation);
    // global 6 = the component the corner EMF uses (Fx[BY] / Fy[BX]), global 7 = Fx[BZ] / Fy[BZ]
    double fb[NM];
    {
      const double cL = inL ? (a.dt / (I.dlf[0][il] * I.dlf[1][jl] * dz)) * (AX == 0 ? I.dlf[1][jl] * dz : I.dlf[0][il] * dz) : 0.;
      const double cR = inR ? (a.dt / (I.dlf[0][i] * I.dlf[1][j] * dz)) * (AX == 0 ? I.dlf[1][j] * dz : I.dlf[0][i] * dz) : 0.;
#pragma unroll
      for (int v = 0; v < 6; ++v) {
        double g = 0.;
        if (inR) g += cR * a.Ub[v * I.sv + f];
        if (inL) g -= cL * a.Ub[v * I.sv + cidx(I, il, jl)];
        // global v -> local position
        fb[AX == 0 ? v : (v == 1 ? VZ : v == 2 ? VX : v == 3 ? VY : v)] = g;
      }
      // bz: -dt/(dx dy) dy (Fx7(i+1) - Fx7(i)) and +dt/(dx dy) dx (ext - exb) with exb = -Fy7
      double g7 = 0.;
      if (inR) g7 += (a.dt / (I.dlf[0][i] * I.dlf[1][j])) * (AX == 0 ? I.dlf[1][j] : I.dlf[0][i]) * bz_total(I, a, i, j);
      if (inL) g7 -= (a.dt / (I.dlf[0][il] * I.dlf[1][jl])) * (AX == 0 ? I.dlf[1][jl] : I.dlf[0][il]) * bz_total(I, a, il, jl);
      // corner EMF: E(ci,cj) = 0.5 (-Fx6(ci,cj-1) - Fx6(ci,cj) + Fy6(ci-1,cj) + Fy6(ci,cj)) - ...
      const double g6 = AX == 0 ? -0.5 * (corner_b(I, a, i, j) + corner_b(I, a, i, j + 1))
                                : 0.5 * (corner_b(I, a, i, j) + corner_b(I, a, i + 1, j));
      fb[BX] = 0.;
      fb[BY] = AX == 0 ? g6 : g7;
      fb[BZ] = AX == 0 ? g7 : g6;
    }
    // face states exactly as the forward builds them
    double wL[NM], wR[NM];
    if (ORDER == 0) {
      double cl_[NM], cr_[NM];
      read_cell(I, a.Wsrc, il, jl, true, cl_);
      read_cell(I, a.Wsrc, i, j, true, cr_);
#pragma unroll
      for (int v = 0; v < NM; ++v) {
        const int gv = plain::perm<AX>(v);
        wL[v] = cl_[gv];
        wR[v] = cr_[gv];
      }
    } else if (CHAR) {
      // projected slopes of the two cells (all nine local variables of the
      // four-cell stencil), as the forward's half_slopes_char
      double c4[4][NM], dL[NM], dR[NM];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int v = 0; v < NM; ++v) c4[q][v] = plm_cell<AX, ORDER>(I, a.Wsrc, i, j, q, plain::perm<AX>(v));
      adj::slopes_char(lim, c4[0], c4[1], c4[2], I.gam, dL);
      adj::slopes_char(lim, c4[1], c4[2], c4[3], I.gam, dR);
#pragma unroll
      for (int v = 0; v < NM; ++v) {
        wL[v] = c4[1][v] + dL[v];
        wR[v] = c4[2][v] - dR[v];
      }
    } else {
#pragma unroll
      for (int v = 0; v < NM; ++v) {
        if (v == BX) continue;
        const int gv = plain::perm<AX>(v);
        const double c0 = plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 0, gv), c1 = plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 1, gv);
        const double c2 = plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 2, gv), c3 = plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 3, gv);
        wL[v] = c1 + plain::half_slope_rt(lim, c0, c1, c2);
        wR[v] = c2 - plain::half_slope_rt(lim, c1, c2, c3);
      }
    }
    const double bn = read_face<AX>(I, a.Bsrc, i, j, ORDER == 0);
    wL[BX] = wR[BX] = bn;
    double wLb[NM], wRb[NM];
#pragma unroll
    for (int v = 0; v < NM; ++v) wLb[v] = wRb[v] = 0.;
    if (RS == dev::RS_HLLD) adj::vjp_hlld(wL, wR, I.gam, fb, wLb, wRb);
    else if (RS == dev::RS_HLLT) adj::vjp_hllt(wL, wR, I.gam, fb, wLb, wRb);
    else adj::vjp_hll(wL, wR, I.gam, fb, wLb, wRb);
    // per-cell contributions, global variable order
    double* Qa = a.Q + (long long)AX * 4 * NM * I.sv;
    if (ORDER == 1 && CHAR) {
      // wL = c1 + d(c0, c1, c2), wR = c2 - d(c1, c2, c3); the face's normal
      // field replaces both BX entries, the cells' own BX still shapes the
      // eigen-system, so all nine entries of the four cells are written
      double c4[4][NM], cb[4][NM], db[NM];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int v = 0; v < NM; ++v) {
          c4[q][v] = plm_cell<AX, ORDER>(I, a.Wsrc, i, j, q, plain::perm<AX>(v));
          cb[q][v] = 0.;
        }
#pragma unroll
      for (int v = 0; v < NM; ++v) {
        const double l = v == BX ? 0. : wLb[v];
        cb[1][v] += l;
        db[v] = l;
      }
      adj::vjp_slopes_char(lim, c4[0], c4[1], c4[2], I.gam, db, cb[0], cb[1], cb[2]);
#pragma unroll
      for (int v = 0; v < NM; ++v) {
        const double r = v == BX ? 0. : wRb[v];
        cb[2][v] += r;
        db[v] = -r;
      }
      adj::vjp_slopes_char(lim, c4[1], c4[2], c4[3], I.gam, db, cb[1], cb[2], cb[3]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int v = 0; v < NM; ++v) Qa[(q * NM + plain::perm<AX>(v)) * I.sv + f] = cb[q][v];
    } else {
#pragma unroll
      for (int v = 0; v < NM; ++v) {
        if (v == BX) continue;
        const int gv = plain::perm<AX>(v);
        if (ORDER == 0) {
          Qa[(1 * NM + gv) * I.sv + f] = wLb[v];
          Qa[(2 * NM + gv) * I.sv + f] = wRb[v];
        } else {
          double c4[4];
          adj::vjp_plm(lim, plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 0, gv), plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 1, gv),
                       plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 2, gv), plm_cell<AX, ORDER>(I, a.Wsrc, i, j, 3, gv), wLb[v],
                       wRb[v], c4);
#pragma unroll
          for (int q = 0; q < 4; ++q) Qa[(q * NM + gv) * I.sv + f] = c4[q];
        }
      }
    }
    // the normal field of the face, and B^n's identity part of the update
    const double bnb = wLb[BX] + wRb[BX];
    const bool out = AX == 0 ? (j >= R.ja && j <= R.jb) : (i >= R.ia && i <= R.ib);
    double vb = out ? face_total<AX>(I, a, i, j) : 0.;
    if (ORDER == 0) vb += bnb;
    else a.Bsrc_b[AX * I.sv + f] = bnb;
    if (vb != 0.) a.Vb[AX * I.sv + f] += vb;
  }
}

// Both face directions in one launch (the x faces first), so the two halves
// share the waves of one grid.
template <int ORDER, int RS, bool CHAR>
__global__ void __launch_bounds__(128, BNZ_ADJ_FACE_MINB) k_faces(const Inst I, const StageArgs a, int lim) {
  int fi0, fj0, w;
  long long nx, ny;
  face_range<0>(a.R, fi0, fj0, w, nx);
  face_range<1>(a.R, fi0, fj0, w, ny);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nx + ny;
       t += (long long)gridDim.x * blockDim.x) {
    if (t < nx) face_vjp<0, ORDER, RS, CHAR>(I, a, lim, t);
    else face_vjp<1, ORDER, RS, CHAR>(I, a, lim, t - nx);
  }
}

// --- S4: per cell read by the stage, the sum over the faces that read it,
// plus the cell-centred EMF's cotangent ---------------------------------------
// With `next` (the corrector's gather, whose cells are exactly the
// predictor's update range), the predictor's S1 runs on the gathered
// cotangent at once instead of a separate launch reading it back.
__global__ void k_gather(const Inst I, const StageArgs a, const StageArgs next, int fuse_next) {
  const Box R = a.R;
  const int h = a.order == 0 ? 1 : 2;
  const int gi0 = R.ia - h, gi1 = R.ib + h, gj0 = R.ja - h, gj1 = R.jb + h;
  const int w = gi1 - gi0 + 1;
  const long long n = (long long)w * (gj1 - gj0 + 1);
  const double* Qx = a.Q;
  const double* Qy = a.Q + 4LL * NM * I.sv;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = gi0 + (int)(t % w), j = gj0 + (int)(t / w);
    double acc[NM];
#pragma unroll
    for (int v = 0; v < NM; ++v) acc[v] = 0.;
    // x faces f (rows ja-1..jb+1, f in ia..ib+1) reading cell i from slot s: f = i + 2 - s
    if (j >= R.ja - 1 && j <= R.jb + 1) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        if (a.order == 0 && (s == 0 || s == 3)) continue;
        const int f = i + 2 - s;
        if (f < R.ia || f > R.ib + 1) continue;
        const long long fc = cidx(I, f, j);
#pragma unroll
        for (int v = 0; v < NM; ++v)
          if (v != BX || a.charact) acc[v] += Qx[(s * NM + v) * I.sv + fc];
      }
    }
    // y faces (columns ia-1..ib+1, rows f in ja..jb+1)
    if (i >= R.ia - 1 && i <= R.ib + 1) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        if (a.order == 0 && (s == 0 || s == 3)) continue;
        const int f = j + 2 - s;
        if (f < R.ja || f > R.jb + 1) continue;
        const long long fc = cidx(I, i, f);
#pragma unroll
        for (int v = 0; v < NM; ++v)
          if (v != BY || a.charact) acc[v] += Qy[(s * NM + v) * I.sv + fc];
      }
    }
    // cell-centred E_z = -(vx by - vy bx) on cells ia-1..ib+1, ja-1..jb+1
    if (i >= R.ia - 1 && i <= R.ib + 1 && j >= R.ja - 1 && j <= R.jb + 1) {
      const double ecb = -0.25 * (corner_b(I, a, i, j) + corner_b(I, a, i + 1, j) + corner_b(I, a, i, j + 1) +
                                  corner_b(I, a, i + 1, j + 1));
      if (ecb != 0.) {
        double wc[NM];
        read_cell(I, a.Wsrc, i, j, a.order == 0, wc);
        acc[VX] -= ecb * wc[BY];
        acc[BY] -= ecb * wc[VX];
        acc[VY] += ecb * wc[BX];
        acc[BX] += ecb * wc[VY];
      }
    }
    const long long c = cidx(I, i, j);
    // the corrector's gravity term reads its stage input ws at updated cells
    // (Ub of this cell is read before the fused predictor S1 below overwrites it)
    if (a.order == 1 && in(R, i, j) && grav_on(I)) {
      double ub[EN + 1];
#pragma unroll
      for (int v = 0; v <= EN; ++v) ub[v] = a.Ub[v * I.sv + c];
      grav_vjp(I, a.dt, ub, a.Wsrc[RHO * I.sv + c], a.Wsrc[VX * I.sv + c], a.Wsrc[VY * I.sv + c],
               a.Wsrc[VZ * I.sv + c], acc);
    }
    // z face (cell-centred in 2D): bz = bz^n + ... on updated cells (reads Ub
    // of this cell before the fused predictor S1 below overwrites it)
    if (in(R, i, j)) a.Vb[2 * I.sv + c] += bz_total(I, a, i, j);
    if (a.order == 0) {
#pragma unroll
      for (int v = 0; v < NM; ++v) a.Vw[v * I.sv + c] += acc[v];
    } else if (fuse_next) {
      cells_body(I, next, i, j, acc);
    } else {
#pragma unroll
      for (int v = 0; v < NM; ++v) a.Wsrc_b[v * I.sv + c] = acc[v];
    }
  }
}

// --- fold: cotangents of reads at virtual positions onto the sources ------
// Field f: 0..8 prim variables, 9..11 face components.  Along axis AX every
// position maps to (source, sign) or to a zeroed boundary face.
template <int AX>
__device__ __forceinline__ int fold_src(const Inst& I, int f, int a, double& sign, bool& zero) {
  const AxisMap m = axis_map(I, AX);
  bool flip = false;
  zero = false;
  int s;
  if (f < NM) {
    s = map_cell(a, m, flip);
    sign = (flip && (AX == 0 ? (f == VX || f == BX) : (f == VY || f == BY))) ? -1. : 1.;
  } else if (f - NM == AX) {
    s = map_face(a, m, flip, zero);
    sign = flip ? -1. : 1.;
  } else {
    s = map_cell(a, m, flip);
    sign = 1.;
  }
  return s;
}

// One thread per remappable position of each field.  A ghost's value moves
// into its source with an atomic add, which is exact whatever the order
// (several ghosts share a source under outflow).
// Both axes at once: every position whose x or y index can be remapped (the
// ghost bands and the first active row / column) sends its value to the source
// both axis maps give it, with the product of the signs; a zeroed face on
// either axis drops it.  Sources are never remappable positions, so one pass
// of atomic adds is exact.
__global__ void k_fold2d(const Inst I, double* Vw, double* Vb) {
  const int a1x = I.ng, a2x = I.ng + I.N[0] - 1, a1y = I.ng, a2y = I.ng + I.N[1] - 1;
  const int rx = a1x + 1 + (I.nx - a2x - 1), ry = a1y + 1 + (I.ny - a2y - 1);
  // band positions: rows j in the y band (all i), then rows outside it with i in the x band
  const long long nband_y = (long long)ry * I.nx;
  const long long nband_x = (long long)(I.ny - ry) * rx;
  const long long per_field = nband_y + nband_x;
  const long long total = 12 * per_field;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(t / per_field);
    const long long u = t - (long long)f * per_field;
    int i, j;
    if (u < nband_y) {
      const int r = (int)(u / I.nx);
      i = (int)(u - (long long)r * I.nx);
      j = r <= a1y ? r : a2y + 1 + (r - a1y - 1);
    } else {
      const long long v = u - nband_y;
      const int r = (int)(v / rx), q = (int)(v - (long long)r * rx);
      j = a1y + 1 + r;  // rows a1y+1 .. a2y
      i = q <= a1x ? q : a2x + 1 + (q - a1x - 1);
    }
    double sx, sy;
    bool zx, zy;
    const int si = fold_src<0>(I, f, i, sx, zx);
    const int sj = fold_src<1>(I, f, j, sy, zy);
    if (si == i && sj == j && !zx && !zy) continue;
    double* V = f < NM ? Vw + (long long)f * I.sv : Vb + (long long)(f - NM) * I.sv;
    const long long p = cidx(I, i, j);
    const double val = V[p];
    V[p] = 0.;
    if (!zx && !zy && val != 0.) atomicAdd(&V[cidx(I, si, sj)], sx * sy * val);
  }
}

}  // namespace adjk
