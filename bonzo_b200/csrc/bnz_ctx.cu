// bnz_ctx.cu -- host side of the C ABI declared in include/bnz_gpu.h.
//
// One context = one grid (BnzGrid + BnzIntegr of the reference): coordinates,
// device state, scratch and the CUDA stream its calls are ordered on.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bnz_ctx_internal.h"

using namespace bnzi;

namespace bnzi {

int fail(bnz_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

// coord.pyx:122-258 (uniform axes) + cartesian.pyx:18-43: face coordinates,
// periodic / reflected ghost spacings, centres and spacings.
void set_coordinates(bnz_ctx* c) {
  for (int n = 0; n < 3; ++n) {
    int Ntot = c->Ntot[n];
    std::vector<double>& lf = c->lf[n];
    lf.assign(Ntot + 1, 0.);
    if (Ntot == 1) {
      lf[0] = c->gd.lmin[n];
      lf[1] = c->gd.lmax[n];
    } else {
      int ind1 = n == 0 ? c->i1 : n == 1 ? c->j1 : c->k1;
      int ind2 = n == 0 ? c->i2 : n == 1 ? c->j2 : c->k2;
      int Nact = ind2 - ind1 + 1;
      double dx = (c->gd.lmax[n] - c->gd.lmin[n]) / Nact;
      double l1 = 0 * Nact * dx;
      for (int i = 0; i < Ntot + 1; ++i) lf[i] = l1 + (i - ind1) * dx;
      int b0 = c->gd.bc[n][0], b1 = c->gd.bc[n][1];
      if (b0 == BNZ_BC_PERIODIC)
        for (int i = ind1 - 1; i > -1; --i) {
          int i_ = ind2 - i + (ind1 - 1);
          double d = lf[i_ + 1] - lf[i_];
          lf[i] = lf[i + 1] - d;
        }
      if (b1 == BNZ_BC_PERIODIC)
        for (int i = ind2 + 1; i < Ntot; ++i) {
          int i_ = ind1 + i - (ind2 + 1);
          double d = lf[i_ + 1] - lf[i_];
          lf[i + 1] = lf[i] + d;
        }
      if (b0 == BNZ_BC_REFLECT)
        for (int i = ind1 - 1; i > -1; --i) {
          int i_ = ind1 - i + (ind1 - 1);
          double d = lf[i_ + 1] - lf[i_];
          lf[i] = lf[i + 1] - d;
        }
      if (b1 == BNZ_BC_REFLECT)
        for (int i = ind2 + 1; i < Ntot; ++i) {
          int i_ = ind2 - i + (ind2 + 1);
          double d = lf[i_ + 1] - lf[i_];
          lf[i + 1] = lf[i] + d;
        }
    }
    c->dlf[n].assign(Ntot, 0.);
    c->dlf_inv[n].assign(Ntot, 0.);
    c->lv[n].assign(Ntot, 0.);
    c->dlv[n].assign(Ntot, 0.);
    c->dlv_inv[n].assign(Ntot, 0.);
    for (int i = 0; i < Ntot; ++i) {
      c->dlf[n][i] = lf[i + 1] - lf[i];
      c->dlf_inv[n][i] = 1. / c->dlf[n][i];
      c->lv[n][i] = 0.5 * (lf[i] + lf[i + 1]);
    }
    for (int i = 1; i < Ntot; ++i) {
      c->dlv[n][i] = c->lv[n][i] - c->lv[n][i - 1];
      c->dlv_inv[n][i] = 1. / c->dlv[n][i];
    }
  }
}

StepArgs step_args(bnz_ctx* c) {
  StepArgs a;
  memset(&a, 0, sizeof a);
  a.g = c->g;
  a.prim = c->prim;
  a.cons = c->cons;
  a.bfld = c->bfld;
  a.cons_s = c->cons_s;
  a.bfld_s = c->bfld_s;
  // unused axes alias the x fluxes (never read there)
  for (int d = 0; d < 3; ++d) a.flx[d] = c->flx[d] ? c->flx[d] : c->flx[0];
  a.ec = c->ec;
  a.ee = c->ee;
  a.wnext = c->wnext;
  a.bnext = c->bnext;
  a.err = c->d_err;
  a.rsolver = c->md.rsolver;
  a.reconstr_order = c->md.reconstr == BNZ_RCN_CONST ? 0 : 1;
  a.limiter = c->md.limiter;
  a.charact_proj = c->md.charact_proj;
  for (int x = 0; x < 3; ++x) {
    a.bc[x][0] = c->gd.bc[x][0];
    a.bc[x][1] = c->gd.bc[x][1];
  }
  a.face_aware = c->md.outflow_face_aware;
  a.stream = c->stream;
  for (int d = 0; d < 3; ++d) a.grav[d] = c->md.grav[d];
  a.fdriv = c->fdriv;
  a.src = src_on(c->md) ? 1 : 0;
  a.hydro = c->md.hydro ? 1 : 0;
  a.smaps = c->d_smaps;
  // the hydro build's HLL takes the hydro sound speed
  if (a.hydro && a.rsolver == BNZ_RS_HLL) a.rsolver = 4;  // dev::RS_HLL_HYDRO
  return a;
}

bool drive_on(const bnz_method_desc& m) { return m.drive_f0 != 0.; }
bool src_on(const bnz_method_desc& m) {
  return m.grav[0] != 0. || m.grav[1] != 0. || m.grav[2] != 0. || drive_on(m);
}

// splitmix64 (Steele, Lea & Flood 2014): the uniform stream behind the driving
// amplitudes (the reference's rand() / RAND_MAX has no reproducible seed)
unsigned long long splitmix64(unsigned long long& st) {
  unsigned long long z = (st += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// turb_driv.pyx:50-79: Gaussian amplitudes c1, c2 of every mode (zero when a
// wavenumber component is zero), Box-Muller from two uniforms
void drive_modes(int nmod, unsigned long long& rng, double* c1, double* c2) {
  const int nmod2 = 2 * nmod + 1;
  for (int p = 0; p < nmod2; ++p)
    for (int q = 0; q < nmod2; ++q)
      for (int r = 0; r < nmod2; ++r)
        for (int n = 0; n < 3; ++n) {
          double norm;
          if (p == nmod || q == nmod || r == nmod) norm = 0.;
          else norm = 1. / ((double)((p - nmod) * (p - nmod)) + (double)((q - nmod) * (q - nmod)) +
                            (double)((r - nmod) * (r - nmod)));
          double w1 = (double)(splitmix64(rng) >> 11) * (1.0 / 9007199254740992.0);
          double w2 = (double)(splitmix64(rng) >> 11) * (1.0 / 9007199254740992.0);
          if (w1 == 0.) w1 = 1e-20;
          const int m = n + 3 * (r + nmod2 * q + nmod2 * nmod2 * p);
          c1[m] = norm * std::sqrt(-2 * std::log(w1)) * std::cos(2 * M_PI * w2);
          c2[m] = norm * std::sqrt(-2 * std::log(w1)) * std::sin(2 * M_PI * w2);
        }
}

// update_physics (integrator.pyx:176-194): new amplitudes, then the force
// field advanced with the dt the device record holds for this step
int drive_advance(bnz_ctx* c) {
  const int nmod = c->md.drive_nmod, nmod2 = 2 * nmod + 1;
  const size_t nc = 3 * (size_t)nmod2 * nmod2 * nmod2;
  CKC(cudaEventSynchronize(c->ev_modes));  // the staging buffer's previous copy is done
  drive_modes(nmod, c->rng, c->h_modes, c->h_modes + nc);
  CKC(cudaMemcpyAsync(c->d_modes, c->h_modes, 2 * nc * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CKC(cudaEventRecord(c->ev_modes, c->stream));
  DriveArgs d;
  d.fdriv = c->fdriv;
  d.modes = c->d_modes;
  d.nmod = nmod;
  for (int a = 0; a < 3; ++a) d.k0[a] = 2. * M_PI / (c->gd.lmax[a] - c->gd.lmin[a]);
  d.tau = c->md.drive_tau;
  d.f0 = c->md.drive_f0;
  c->launches += c->L->drive(step_args(c), d, &c->d_ds->dt);
  CKC(cudaGetLastError());
  return BNZ_OK;
}

void free_all(bnz_ctx* c) {
  // every device buffer exactly once (the fused path aliases prim/bfld with its ping-pong pair)
  double* bufs[] = {c->d_coord, c->prim, c->cons, c->bfld, c->cons_s, c->bfld_s, c->flx[0], c->flx[1], c->flx[2],
                    c->ec, c->ee, c->wnext, c->bnext, c->dscr, c->d_sts, c->wbuf[0], c->wbuf[1], c->bbuf[0],
                    c->bbuf[1]};
  const int nb = sizeof bufs / sizeof bufs[0];
  for (int q = 0; q < nb; ++q) {
    if (!bufs[q]) continue;
    bool seen = false;
    for (int r = 0; r < q; ++r) seen |= bufs[r] == bufs[q];
    if (!seen) cudaFree(bufs[q]);
  }
  c->d_coord = c->prim = c->cons = c->bfld = c->cons_s = c->bfld_s = c->ec = c->ee = nullptr;
  c->wnext = c->bnext = c->dscr = c->d_sts = nullptr;
  for (int d = 0; d < 3; ++d) c->flx[d] = nullptr;
  c->wbuf[0] = c->wbuf[1] = c->bbuf[0] = c->bbuf[1] = nullptr;
  if (c->fdriv) cudaFree(c->fdriv);
  if (c->d_modes) cudaFree(c->d_modes);
  if (c->h_modes) cudaFreeHost(c->h_modes);
  if (c->ev_modes) cudaEventDestroy(c->ev_modes);
  c->fdriv = c->d_modes = c->h_modes = nullptr;
  c->ev_modes = nullptr;
  if (c->d_err) cudaFree(c->d_err);
  if (c->d_ds) cudaFree(c->d_ds);
  if (c->d_inst) cudaFree(c->d_inst);
  if (c->d_tiles) cudaFree(c->d_tiles);
  c->d_inst = nullptr;
  c->d_tiles = nullptr;
  if (c->d_inst3) cudaFree(c->d_inst3);
  if (c->d_tiles3) cudaFree(c->d_tiles3);
  if (c->d_map3) cudaFree(c->d_map3);
  if (c->d_smaps) cudaFree(c->d_smaps);
  c->d_inst3 = nullptr;
  c->d_tiles3 = nullptr;
  c->d_map3 = nullptr;
  c->d_smaps = nullptr;
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
  c->d_err = nullptr;
  c->d_ds = nullptr;
  c->graph = nullptr;
  c->stream = nullptr;
}

// The fused kernels cover 2D and 3D grids with PLM (the corrector is order 1).
bool fused_available(const bnz_grid_desc* g, const bnz_method_desc* m) {
  return (g->dims == 2 || g->dims == 3) && m->reconstr == BNZ_RCN_LINEAR && !m->hydro;
}

void make_tiles3(int inst, const int* N, int ng, bool pred, int tx, int ty, int kz, std::vector<FusedTile3>& out) {
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = pred ? 1 : ng;
    hi[a] = pred ? N[a] + 2 * ng - 2 : ng + N[a] - 1;
  }
  // about kz planes per chunk, the chunks of a column of equal depth
  const int nz = hi[2] - lo[2] + 1, nch = (nz + kz - 1) / kz, cz = (nz + nch - 1) / nch;
  for (int z = lo[2]; z <= hi[2]; z += cz)
    for (int y = lo[1]; y <= hi[1]; y += ty)
      for (int x = lo[0]; x <= hi[0]; x += tx) {
        FusedTile3 t;
        t.inst = inst;
        t.x0 = x;
        t.y0 = y;
        t.z0 = z;
        t.wx = std::min(tx, hi[0] - x + 1);
        t.wy = std::min(ty, hi[1] - y + 1);
        t.wz = std::min(cz, hi[2] - z + 1);
        t.tma = 0;
        out.push_back(t);
      }
}

FusedInst3 make_inst3(const bnz_ctx* c) {
  FusedInst3 I;
  memset(&I, 0, sizeof I);
  I.nx = c->Ntot[0];
  I.ny = c->Ntot[1];
  I.nz = c->Ntot[2];
  I.N[0] = c->i2 - c->i1 + 1;
  I.N[1] = c->j2 - c->j1 + 1;
  I.N[2] = c->k2 - c->k1 + 1;
  I.ng = c->ng;
  I.sv = (long long)c->ncell;
  I.gam = c->md.gam;
  for (int a = 0; a < 3; ++a) {
    I.bc[a][0] = c->gd.bc[a][0];
    I.bc[a][1] = c->gd.bc[a][1];
    I.dlf[a] = c->g.dlf[a];
    I.dlf_inv[a] = c->g.dlf_inv[a];
    I.lf[a] = c->g.lf[a];
    I.lv[a] = c->g.lv[a];
  }
  I.face_aware = c->md.outflow_face_aware;
  I.w[0] = c->wbuf[0];
  I.w[1] = c->wbuf[1];
  I.b[0] = c->bbuf[0];
  I.b[1] = c->bbuf[1];
  I.ws = c->cons_s;
  I.bs = c->bfld_s;
  I.ds = c->d_ds;
  I.err = c->d_err;
  for (int d = 0; d < 3; ++d) I.grav[d] = c->md.grav[d];
  I.fdriv = c->fdriv;
  I.src = src_on(c->md) ? 1 : 0;
  return I;
}

Fused3Launch fused3_launch(const bnz_ctx* c, int dt_mode) {
  Fused3Launch f;
  memset(&f, 0, sizeof f);
  f.insts = c->d_inst3;
  f.ninst = 1;
  f.tilesA = c->d_tiles3;
  f.ntA = c->ntA3;
  f.tilesB = c->d_tiles3 + c->ntA3;
  f.ntB = c->ntB3;
  f.rsolver = c->md.rsolver;
  f.limiter = c->md.limiter;
  f.charact_proj = c->md.charact_proj;
  f.cour = c->md.cour;
  f.dt_mode = dt_mode;
  f.dt_fixed = c->md.dt_fixed;
  f.wsmaps = c->d_map3;
  f.stream = c->stream;
  return f;
}

// Tiles of tx x ty cells over the active range; the predictor's edge tiles
// also cover the two ghost rings it updates (cells 1..Ntot-2).
void make_tiles(int inst, int N0, int N1, int ng, bool pred, int tx, int ty, std::vector<FusedTile>& out) {
  const int T[2] = {tx, ty};
  const int N[2] = {N0, N1};
  int nt[2];
  for (int a = 0; a < 2; ++a) nt[a] = (N[a] + T[a] - 1) / T[a];
  for (int ty = 0; ty < nt[1]; ++ty)
    for (int tx = 0; tx < nt[0]; ++tx) {
      int lo[2], hi[2];  // inclusive, array coordinates
      const int t[2] = {tx, ty};
      for (int a = 0; a < 2; ++a) {
        lo[a] = ng + t[a] * T[a];
        hi[a] = std::min(ng + (t[a] + 1) * T[a], ng + N[a]) - 1;
        if (pred) {
          if (t[a] == 0) lo[a] = 1;
          if (t[a] == nt[a] - 1) hi[a] = N[a] + 2 * ng - 2;
        }
      }
      FusedTile ft;
      ft.inst = inst;
      ft.x0 = lo[0];
      ft.y0 = lo[1];
      ft.wx = hi[0] - lo[0] + 1;
      ft.wy = hi[1] - lo[1] + 1;
      ft.tma = 0;
      out.push_back(ft);
    }
}

// Predictor tiles of the persistent predictor: the predictor range (cells 1 ..
// Ntot-2 of each axis) in plain tx x ty steps from cell 1, so no tile is
// larger than tx x ty.
void make_tiles_uniform(int inst, int N0, int N1, int ng, int tx, int ty, std::vector<FusedTile>& out) {
  const int hi0 = N0 + 2 * ng - 2, hi1 = N1 + 2 * ng - 2;
  for (int y = 1; y <= hi1; y += ty)
    for (int x = 1; x <= hi0; x += tx) {
      FusedTile ft;
      ft.inst = inst;
      ft.x0 = x;
      ft.y0 = y;
      ft.wx = std::min(tx, hi0 - x + 1);
      ft.wy = std::min(ty, hi1 - y + 1);
      ft.tma = 0;
      out.push_back(ft);
    }
}

FusedInst make_inst(const bnz_ctx* c) {
  FusedInst I;
  memset(&I, 0, sizeof I);
  I.nx = c->Ntot[0];
  I.ny = c->Ntot[1];
  I.N[0] = c->i2 - c->i1 + 1;
  I.N[1] = c->j2 - c->j1 + 1;
  I.ng = c->ng;
  I.sv = (long long)c->ncell;
  I.gam = c->md.gam;
  for (int a = 0; a < 2; ++a) {
    I.bc[a][0] = c->gd.bc[a][0];
    I.bc[a][1] = c->gd.bc[a][1];
    I.dlf[a] = c->g.dlf[a];
    I.dlf_inv[a] = c->g.dlf_inv[a];
    I.lf[a] = c->g.lf[a];
    I.lv[a] = c->g.lv[a];
  }
  I.face_aware = c->md.outflow_face_aware;
  I.dlf2 = c->dlf[2][0];
  I.w[0] = c->wbuf[0];
  I.w[1] = c->wbuf[1];
  I.b[0] = c->bbuf[0];
  I.b[1] = c->bbuf[1];
  I.ws = c->cons_s;
  I.bs = c->bfld_s;
  I.ds = c->d_ds;
  I.err = c->d_err;
  for (int d = 0; d < 3; ++d) I.grav[d] = c->md.grav[d];
  I.fdriv = c->fdriv;
  I.src = src_on(c->md) ? 1 : 0;
  return I;
}

int ensure_ghosts(bnz_ctx* c);
int refresh_cds(bnz_ctx* c);

FusedLaunch fused_launch(const bnz_ctx* c, int dt_mode) {
  FusedLaunch f;
  memset(&f, 0, sizeof f);
  f.insts = c->d_inst;
  f.ninst = 1;
  f.tilesA = c->d_tiles;
  f.ntA = c->ntA;
  f.tilesB = c->d_tiles + c->ntA;
  f.ntB = c->ntB;
  f.rsolver = c->md.rsolver;
  f.limiter = c->md.limiter;
  f.charact_proj = c->md.charact_proj;
  f.variant = c->variant;
  f.cour = c->md.cour;
  f.dt_mode = dt_mode;
  f.dt_fixed = c->md.dt_fixed;
  f.err = c->d_err;
  f.stream = c->stream;
  return f;
}

// The 3D context's chunk lists, instance record and the tensor map of ws.
cudaError_t build_ctx3(bnz_ctx* c) {
  std::vector<FusedTile3> t;
  const int N[3] = {c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->k2 - c->k1 + 1};
  make_tiles3(0, N, c->ng, true, F3_TX, F3_TY, F3_KZ, t);
  c->ntA3 = (int)t.size();
  make_tiles3(0, N, c->ng, false, F3_TX, F3_TY, F3_KZ, t);
  c->ntB3 = (int)t.size() - c->ntA3;
  CUtensorMap m;
  const bool ok = ws_map3(c, c->cons_s, &m);
  for (size_t q = c->ntA3; q < t.size(); ++q) t[q].tma = ok ? 1 : 0;
  cudaError_t e = cudaSuccess;
  if (ok) {
    e = cudaMalloc((void**)&c->d_map3, sizeof m);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_map3, &m, sizeof m, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_tiles3, t.size() * sizeof(FusedTile3));
  if (e == cudaSuccess) e = cudaMemcpy(c->d_tiles3, t.data(), t.size() * sizeof(FusedTile3), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_inst3, sizeof(FusedInst3));
  if (e == cudaSuccess) {
    FusedInst3 I = make_inst3(c);
    e = cudaMemcpy(c->d_inst3, &I, sizeof I, cudaMemcpyHostToDevice);
  }
  return e;
}

// (Re)build the single-grid tile lists for the context's variant.
cudaError_t build_ctx_tiles(bnz_ctx* c) {
  const FusedVariant& v = FUSED_VARIANTS[c->variant];
  std::vector<FusedTile> tiles;
  make_tiles(0, c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->ng, true, v.tx, v.ty, tiles);
  c->ntA = (int)tiles.size();
  make_tiles(0, c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->ng, false, v.tx, v.ty, tiles);
  c->ntB = (int)tiles.size() - c->ntA;
  if (c->d_tiles) cudaFree(c->d_tiles);
  c->d_tiles = nullptr;
  cudaError_t e = cudaMalloc((void**)&c->d_tiles, tiles.size() * sizeof(FusedTile));
  if (e == cudaSuccess)
    e = cudaMemcpy(c->d_tiles, tiles.data(), tiles.size() * sizeof(FusedTile), cudaMemcpyHostToDevice);
  return e;
}

int validate(const bnz_grid_desc* g, const bnz_method_desc* m, std::string& why) {
  if (g->dims < 1 || g->dims > 3) return why = "dims must be 1, 2 or 3", 0;
  if (g->Nx < 1 || (g->dims >= 2 && g->Ny < 1) || (g->dims >= 3 && g->Nz < 1)) return why = "grid size < 1", 0;
  if (g->dims < 2 && g->Ny != 1) return why = "cannot set Ny>1 without second dimension", 0;
  if (g->dims < 3 && g->Nz != 1) return why = "cannot set Nz>1 without third dimension", 0;
  for (int a = 0; a < g->dims; ++a) {
    if (!(g->lmax[a] > g->lmin[a])) return why = "lmax must exceed lmin", 0;
    for (int s = 0; s < 2; ++s)
      if (g->bc[a][s] < 0 || g->bc[a][s] > 2) return why = "bc flag must be 0 (periodic), 1 (outflow) or 2 (reflect)", 0;
    if ((g->bc[a][0] == BNZ_BC_PERIODIC) != (g->bc[a][1] == BNZ_BC_PERIODIC))
      return why = "periodic boundaries must be set on both sides of an axis", 0;
  }
  if (!(m->gam > 1.)) return why = "gam must exceed 1", 0;
  if (!(m->cour > 0.)) return why = "cour must be positive", 0;
  if (m->hydro != 0 && m->hydro != 1) return why = "hydro must be 0 or 1", 0;
  if (m->hydro) {
    // the reference's hydro build (MFIELD 0, src/defs_c.h:72-96): hll or hllc
    if (m->rsolver != BNZ_RS_HLL && m->rsolver != BNZ_RS_HLLC)
      return why = "rsolver must be hll or hllc in hydro mode (hlld needs a magnetic field)", 0;
    if (m->path == BNZ_PATH_FUSED) return why = "hydro mode runs on the plain path or the split path", 0;
    if (m->charact_proj) return why = "charact_proj is not available in hydro mode", 0;
    if (m->kappa0 != 0.) return why = "field-aligned conduction needs a magnetic field (kappa0 = 0 in hydro mode)", 0;
  } else if (m->rsolver != BNZ_RS_HLL && m->rsolver != BNZ_RS_HLLD && m->rsolver != BNZ_RS_HLLT) {
    return why = "rsolver must be hll, hlld or hllt for MHD (hllc is hydro-only in the reference; set hydro = 1)", 0;
  }
  if (m->reconstr != BNZ_RCN_CONST && m->reconstr != BNZ_RCN_LINEAR) return why = "reconstr must be const or linear", 0;
  if (m->limiter < 0 || m->limiter > 2) return why = "limiter must be vl, mc or mm", 0;
  if (m->charact_proj != 0 && m->charact_proj != 1) return why = "charact_proj must be 0 or 1", 0;
  if (m->drive_f0 != 0.) {
    if (!(m->drive_tau > 0.)) return why = "tau must be positive when the driving is on", 0;
    if (m->drive_nmod < 1 || m->drive_nmod > 8) return why = "nmod must be 1..8", 0;
  }
  if (m->kappa0 < 0.) return why = "kappa0 must be >= 0", 0;
  if (m->kappa0 > 0. && !(m->cour_diff > 0.)) return why = "cour_diff must be positive", 0;
  if (m->path != BNZ_PATH_FUSED && m->path != BNZ_PATH_PLAIN && m->path != BNZ_PATH_SPLIT)
    return why = "path must be fused, plain or split", 0;
  if (m->path == BNZ_PATH_FUSED && !fused_available(g, m)) return why = "fused path not available for this grid", 0;
  int ng = m->reconstr == BNZ_RCN_CONST ? 2 : 3;
  int N[3] = {g->Nx, g->Ny, g->Nz};
  for (int a = 0; a < g->dims; ++a)
    if (N[a] < ng) return why = "each active axis needs at least ng cells", 0;
  return 1;
}

}  // namespace bnzi

namespace {

// Pull the device time record into the host copy after graph stepping.
int sync_time(bnz_ctx* c) {
  if (!c->time_on_device) return BNZ_OK;
  DtState ds;
  CKC(cudaMemcpyAsync(&ds, c->d_ds, sizeof ds, cudaMemcpyDeviceToHost, c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  c->time = ds.time;
  c->step = (long)ds.step;
  c->last_dt = ds.dt;
  c->time_on_device = false;
  return BNZ_OK;
}

}  // namespace

extern "C" {

int bnz_create(const bnz_grid_desc* gd, const bnz_method_desc* md, bnz_ctx** out) {
  if (!gd || !md || !out) return BNZ_ERR_ARG;
  *out = nullptr;
  std::string why;
  bnz_ctx* c = new bnz_ctx();
  if (!validate(gd, md, why)) {
    // a context is still returned so that bnz_last_error can report why
    c->err = why;
    *out = c;
    return BNZ_ERR_ARG;
  }
  c->gd = *gd;
  c->md = *md;
  c->ng = md->reconstr == BNZ_RCN_CONST ? 2 : 3;
  int dims = gd->dims, ng = c->ng;
  int Na[3] = {gd->Nx, dims >= 2 ? gd->Ny : 1, dims >= 3 ? gd->Nz : 1};
  for (int a = 0; a < 3; ++a) c->Ntot[a] = a < dims ? Na[a] + 2 * ng : 1;
  c->i1 = ng;
  c->i2 = Na[0] + ng - 1;
  c->j1 = dims >= 2 ? ng : 0;
  c->j2 = dims >= 2 ? Na[1] + ng - 1 : 0;
  c->k1 = dims >= 3 ? ng : 0;
  c->k2 = dims >= 3 ? Na[2] + ng - 1 : 0;
  c->ncell = (size_t)c->Ntot[0] * c->Ntot[1] * c->Ntot[2];
  set_coordinates(c);
  c->L = md->exact_fp ? &exact::table : &fast::table;

  cudaError_t e;
#define ALLOC(ptr, bytes)                                                                      \
  do {                                                                                         \
    e = cudaMalloc((void**)&(ptr), (bytes));                                                   \
    if (e != cudaSuccess) {                                                                    \
      int code = e == cudaErrorMemoryAllocation ? BNZ_ERR_NOMEM : BNZ_ERR_CUDA;                \
      c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);                            \
      free_all(c);                                                                             \
      *out = c;                                                                                \
      return code;                                                                             \
    }                                                                                          \
  } while (0)

  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    c->err = std::string("cudaStreamCreate: ") + cudaGetErrorString(e);
    *out = c;
    return BNZ_ERR_CUDA;
  }
  // coordinates: 5 arrays per axis, each Ntot+1 long
  size_t ncoord = 0;
  for (int a = 0; a < 3; ++a) ncoord += 5 * (size_t)(c->Ntot[a] + 1);
  ALLOC(c->d_coord, ncoord * sizeof(double));
  {
    std::vector<double> h(ncoord, 0.);
    size_t off = 0;
    const double* ptrs[3][5];
    for (int a = 0; a < 3; ++a) {
      const std::vector<double>* src[5] = {&c->dlf[a], &c->dlf_inv[a], &c->lf[a], &c->lv[a], &c->dlv_inv[a]};
      for (int q = 0; q < 5; ++q) {
        std::copy(src[q]->begin(), src[q]->end(), h.begin() + off);
        ptrs[a][q] = c->d_coord + off;
        off += c->Ntot[a] + 1;
      }
    }
    e = cudaMemcpy(c->d_coord, h.data(), ncoord * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      c->err = std::string("cudaMemcpy: ") + cudaGetErrorString(e);
      free_all(c);
      *out = c;
      return BNZ_ERR_CUDA;
    }
    GridDev& g = c->g;
    g.nx = c->Ntot[0];
    g.ny = c->Ntot[1];
    g.nz = c->Ntot[2];
    g.dims = dims;
    g.ng = ng;
    g.i1 = c->i1; g.i2 = c->i2; g.j1 = c->j1; g.j2 = c->j2; g.k1 = c->k1; g.k2 = c->k2;
    g.sv = (long long)c->ncell;
    g.gam = md->gam;
    for (int a = 0; a < 3; ++a) {
      g.dlf[a] = ptrs[a][0];
      g.dlf_inv[a] = ptrs[a][1];
      g.lf[a] = ptrs[a][2];
      g.lv[a] = ptrs[a][3];
      g.dlv_inv[a] = ptrs[a][4];
    }
  }
  size_t n9 = 9 * c->ncell * sizeof(double), n3 = 3 * c->ncell * sizeof(double);
  ALLOC(c->prim, n9);
  ALLOC(c->cons, n9);
  ALLOC(c->bfld, n3);
  if (md->path != BNZ_PATH_FUSED) {
    // plain and split paths; the split path keeps the step's b^n in ec
    ALLOC(c->cons_s, n9);
    ALLOC(c->bfld_s, n3);
    for (int d = 0; d < dims; ++d) ALLOC(c->flx[d], n9);
    ALLOC(c->ec, n3);
    ALLOC(c->ee, n3);
  } else {
    ALLOC(c->wnext, n9);
    ALLOC(c->bnext, n3);
    ALLOC(c->cons_s, n9);   // predictor prim ws
    ALLOC(c->bfld_s, n3);   // predictor faces bs
    c->wbuf[0] = c->prim;
    c->wbuf[1] = c->wnext;
    c->bbuf[0] = c->bfld;
    c->bbuf[1] = c->bnext;
  }
  if (md->kappa0 > 0.) {
    ALLOC(c->dscr, 8 * c->ncell * sizeof(double));
    double* p = c->dscr;
    c->da.temp = p;
    c->da.fx = p + c->ncell;
    c->da.fy = p + 2 * c->ncell;
    c->da.fz = p + 3 * c->ncell;
    c->da.pres0 = p + 4 * c->ncell;
    c->da.presm1 = p + 5 * c->ncell;
    c->da.dtemp = p + 6 * c->ncell;
    c->da.dtemp0 = p + 7 * c->ncell;
    c->da.kappa0 = md->kappa0;
    c->da.aniso = md->thcond_type == BNZ_TC_ANISO;
    c->da.sat = md->sat_hfe;
    c->da.cour_diff = md->cour_diff;
    e = cudaMemsetAsync(c->dscr, 0, 8 * c->ncell * sizeof(double), c->stream);
  }
  if (drive_on(*md)) {
    const int nmod2 = 2 * md->drive_nmod + 1;
    const size_t nm = 2 * 3 * (size_t)nmod2 * nmod2 * nmod2;
    ALLOC(c->fdriv, 3 * c->ncell * sizeof(double));
    ALLOC(c->d_modes, nm * sizeof(double));
    e = cudaMallocHost((void**)&c->h_modes, nm * sizeof(double));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_modes, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->fdriv, 0, 3 * c->ncell * sizeof(double), c->stream);
    c->rng = md->drive_seed;
  }
  e = cudaMalloc((void**)&c->d_err, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_ds, sizeof(DtState));
  if (e == cudaSuccess && md->path == BNZ_PATH_SPLIT && dims == 3) {
    e = build_split_maps(c);
  } else if (e == cudaSuccess && md->path == BNZ_PATH_FUSED && dims == 3) {
    e = build_ctx3(c);
  } else if (e == cudaSuccess && md->path == BNZ_PATH_FUSED) {
    e = build_ctx_tiles(c);
    if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_inst, sizeof(FusedInst));
    if (e == cudaSuccess) {
      FusedInst I = make_inst(c);
      e = cudaMemcpy(c->d_inst, &I, sizeof I, cudaMemcpyHostToDevice);
    }
  }
  if (e != cudaSuccess) {
    c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    free_all(c);
    *out = c;
    return BNZ_ERR_NOMEM;
  }
  cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream);
  cudaMemsetAsync(c->d_ds, 0, sizeof(DtState), c->stream);
  cudaMemsetAsync(c->prim, 0, n9, c->stream);
  cudaMemsetAsync(c->cons, 0, n9, c->stream);
  cudaMemsetAsync(c->bfld, 0, n3, c->stream);
  if (c->cons_s) cudaMemsetAsync(c->cons_s, 0, n9, c->stream);
  if (c->bfld_s) cudaMemsetAsync(c->bfld_s, 0, n3, c->stream);
  if (c->wnext) cudaMemsetAsync(c->wnext, 0, n9, c->stream);
  if (c->bnext) cudaMemsetAsync(c->bnext, 0, n3, c->stream);
  for (int d = 0; d < dims; ++d)
    if (c->flx[d]) cudaMemsetAsync(c->flx[d], 0, n9, c->stream);
  e = cudaStreamSynchronize(c->stream);
  *out = c;
  if (e != cudaSuccess) return fail(c, BNZ_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
  return BNZ_OK;
#undef ALLOC
}

int bnz_destroy(bnz_ctx* c) {
  if (!c) return BNZ_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  adj_free(c);
  io_free(c);
  free_all(c);
  delete c;
  return BNZ_OK;
}

const char* bnz_last_error(const bnz_ctx* c) { return c ? c->err.c_str() : "null context"; }

int bnz_shape(const bnz_ctx* c, int* ntot, int* ng) {
  if (!c) return BNZ_ERR_ARG;
  if (ntot)
    for (int a = 0; a < 3; ++a) ntot[a] = c->Ntot[a];
  if (ng) *ng = c->ng;
  return BNZ_OK;
}

int bnz_set_state(bnz_ctx* c, const double* pc, int is_prim, const double* bfld) {
  if (!c || !pc) return fail(c, BNZ_ERR_ARG, "null state pointer");
  if (!c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  size_t n9 = 9 * c->ncell * sizeof(double), n3 = 3 * c->ncell * sizeof(double);
  CKC(cudaMemcpyAsync(is_prim ? c->prim : c->cons, pc, n9, cudaMemcpyHostToDevice, c->stream));
  if (bfld) CKC(cudaMemcpyAsync(c->bfld, bfld, n3, cudaMemcpyHostToDevice, c->stream));
  if (c->md.hydro) {
    // no magnetic field in the hydro build: the field entries are zero
    CKC(cudaMemsetAsync((is_prim ? c->prim : c->cons) + 6 * c->ncell, 0, 3 * c->ncell * sizeof(double), c->stream));
    CKC(cudaMemsetAsync(c->bfld, 0, n3, c->stream));
  }
  // derive the other array on every cell, as init_sim does after set_problem
  StepArgs a = step_args(c);
  if (is_prim) c->launches += c->L->prim2cons_all(a);
  else c->launches += c->L->cons2prim_all(a);
  c->ghosts_stale = false;
  c->cons_stale = false;
  int rc = refresh_cds(c);
  if (rc) return rc;
  CKC(cudaGetLastError());
  CKC(cudaStreamSynchronize(c->stream));
  return BNZ_OK;
}

int bnz_init(bnz_ctx* c) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  StepArgs a = step_args(c);
  c->launches += c->L->apply_bc(a, c->prim, c->bfld, 0xFFFu);
  c->launches += c->L->interp_bc_active(a);
  c->launches += c->L->apply_bc(a, c->prim, c->bfld, (1u << 6) | (1u << 7) | (1u << 8));
  c->launches += c->L->prim2cons_all(a);
  DtState ds;
  memset(&ds, 0, sizeof ds);
  CKC(cudaMemcpyAsync(c->d_ds, &ds, sizeof ds, cudaMemcpyHostToDevice, c->stream));
  c->ghosts_stale = false;
  c->cons_stale = false;
  int rc = refresh_cds(c);
  if (rc) return rc;
  CKC(cudaGetLastError());
  CKC(cudaStreamSynchronize(c->stream));
  c->time = 0.;
  c->step = 0;
  c->time_on_device = false;
  return BNZ_OK;
}

int bnz_get_state(bnz_ctx* c, double* prim, double* cons, double* bfld) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  int rc = ensure_ghosts(c);
  if (rc) return rc;
  size_t n9 = 9 * c->ncell * sizeof(double), n3 = 3 * c->ncell * sizeof(double);
  if (prim) CKC(cudaMemcpyAsync(prim, c->prim, n9, cudaMemcpyDeviceToHost, c->stream));
  if (cons) CKC(cudaMemcpyAsync(cons, c->cons, n9, cudaMemcpyDeviceToHost, c->stream));
  if (bfld) CKC(cudaMemcpyAsync(bfld, c->bfld, n3, cudaMemcpyDeviceToHost, c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  return BNZ_OK;
}

int bnz_apply_bc(bnz_ctx* c, uint32_t mask) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (mask & ~0xFFFu) return fail(c, BNZ_ERR_ARG, "var_mask has bits above 11");
  int rc = ensure_ghosts(c);
  if (rc) return rc;
  StepArgs a = step_args(c);
  c->launches += c->L->apply_bc(a, c->prim, c->bfld, mask);
  CKC(cudaGetLastError());
  return BNZ_OK;
}

int bnz_new_dt(bnz_ctx* c, double* dt_out) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  StepArgs a = step_args(c);
  c->launches += c->L->new_dt(a, c->prim, c->d_ds, c->md.cour, 0);
  CKC(cudaGetLastError());
  DtState ds;
  CKC(cudaMemcpyAsync(&ds, c->d_ds, sizeof ds, cudaMemcpyDeviceToHost, c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  if (dt_out) *dt_out = ds.dt;
  return BNZ_OK;
}

}  // extern "C"

namespace bnzi {

// RKL2 stage loop (thcond_elec.pyx:17-113); dtp points at the hyperbolic dt.
int diffuse_impl(bnz_ctx* c, const double* dtp, double dt_hyp, int* nsts_out) {
  if (c->md.kappa0 == 0.) {
    if (nsts_out) *nsts_out = 0;
    return BNZ_OK;
  }
  StepArgs a = step_args(c);
  c->launches += c->L->apply_bc(a, c->prim, c->bfld, 0xFFFu);
  // diffusive dt: max over active cells, read back to size the stage loop
  unsigned long long* slot = &c->d_ds->cdsmax_bits;
  CKC(cudaMemsetAsync(slot, 0, sizeof(unsigned long long), c->stream));
  c->launches += c->L->diff_dt_max(a, c->da, slot);
  unsigned long long bits = 0;
  CKC(cudaMemcpyAsync(&bits, slot, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  double mx;
  memcpy(&mx, &bits, sizeof mx);
  double dt_diff = c->md.cour_diff / mx;
  // diffusion.pyx:217-224
  int s = dt_diff >= dt_hyp ? 1 : (int)(0.5 * (std::sqrt(9. + 16. * dt_hyp / dt_diff) - 1.)) + 1;
  // diffusion.pyx:227-260, columns MU NU MUT GAMT
  std::vector<double> cf((size_t)(s + 1) * 4, 0.);
  if (s == 1) {
    cf[4 + 2] = 1.;
  } else {
    std::vector<double> b(s + 1, 0.);
    double one3rd = 1. / 3;
    double w1 = 4. / (s * s + s - 2);
    b[0] = one3rd;
    b[1] = one3rd;
    cf[4 + 2] = w1 * b[1];
    for (int j = 2; j <= s; ++j) {
      b[j] = (double)(j * j + j - 2) / (2 * j * (j + 1));
      cf[j * 4 + 0] = (double)(2 * j - 1) / j * b[j] / b[j - 1];
      cf[j * 4 + 1] = (1. - j) / j * b[j] / b[j - 2];
      cf[j * 4 + 2] = w1 * cf[j * 4 + 0];
      cf[j * 4 + 3] = (b[j - 1] - 1) * cf[j * 4 + 2];
    }
  }
  c->last_nsts = s;
  if (nsts_out) *nsts_out = s;
  for (int n = 1; n <= s; ++n) {
    c->launches += c->L->diff_stage(a, c->da, n == 1, &cf[(size_t)n * 4], dtp);
    if (n % c->ng == 0 && n != s) c->L->apply_bc(a, c->prim, c->bfld, 1u << 4);
  }
  CKC(cudaGetLastError());
  return BNZ_OK;
}

// Fill ghosts and cons of the fused path's current state, or cons of the split
// path's (what the reference's end-of-step BC + prim2cons leave behind,
// vanleer.pyx:162-163).
int ensure_ghosts(bnz_ctx* c) {
  if (!c->ghosts_stale && !c->cons_stale) return BNZ_OK;
  StepArgs a = step_args(c);
  if (c->ghosts_stale) c->launches += c->L->apply_bc(a, c->prim, c->bfld, 0xFFFu);
  c->launches += c->L->prim2cons_all(a);
  CKC(cudaGetLastError());
  c->ghosts_stale = false;
  c->cons_stale = false;
  return BNZ_OK;
}

// CFL max of the current state into the fused slot of the current parity.
int refresh_cds(bnz_ctx* c) {
  if (c->md.path != BNZ_PATH_FUSED) return BNZ_OK;
  CKC(cudaMemsetAsync(&c->d_ds->cds_bits[c->parity], 0, sizeof(unsigned long long), c->stream));
  if (c->gd.dims == 3) c->launches += c->L->fused3_cds(fused3_launch(c, FDT_EXPLICIT), c->parity);
  else c->launches += c->L->fused_cds(fused_launch(c, FDT_EXPLICIT), c->parity);
  CKC(cudaGetLastError());
  return BNZ_OK;
}

void set_parity(bnz_ctx* c, int p) {
  c->parity = p;
  c->prim = c->wbuf[p];
  c->bfld = c->bbuf[p];
}

// vanleer.pyx:101-163 with dt already in d_ds->dt.  dt_mode selects how the
// fused path obtains dt (explicit host value, device CFL, or FIXDT).
int step_impl(bnz_ctx* c, double dt_host, int dt_mode) {
  if (drive_on(c->md)) {
    // the force needs this step's dt in the device record before the stages
    if (dt_mode != FDT_EXPLICIT) return fail(c, BNZ_ERR_UNSUPPORTED, "driving needs the host dt of each step");
    int rc = drive_advance(c);
    if (rc) return rc;
  }
  StepArgs a = step_args(c);
  const double* dtp = &c->d_ds->dt;
  if (c->md.path == BNZ_PATH_PLAIN) {
    c->launches += c->L->plain_predictor_corrector(a, dtp);
  } else if (c->md.path == BNZ_PATH_SPLIT) {
    c->launches += c->L->split_predictor_corrector(a, dtp);
  } else {
    if (c->gd.dims == 3) c->launches += c->L->fused3_step(fused3_launch(c, dt_mode), c->parity);
    else c->launches += c->L->fused_step(fused_launch(c, dt_mode), c->parity);
    set_parity(c, c->parity ^ 1);
    c->ghosts_stale = true;
    a = step_args(c);
  }
  CKC(cudaGetLastError());
  if (c->md.kappa0 > 0.) {
    int rc = diffuse_impl(c, dtp, dt_host, nullptr);
    if (rc) return rc;
    if (c->md.path == BNZ_PATH_FUSED) {
      rc = refresh_cds(c);
      if (rc) return rc;
    }
  }
  if (c->md.path != BNZ_PATH_FUSED) c->launches += c->L->apply_bc(a, c->prim, c->bfld, 0xFFFu);
  // vanleer.pyx:162-163; the split path reads no conserved state, so it forms
  // cons when it is asked for
  if (c->md.path == BNZ_PATH_PLAIN) c->launches += c->L->prim2cons_all(a);
  if (c->md.path == BNZ_PATH_SPLIT) c->cons_stale = true;
  CKC(cudaGetLastError());
  return BNZ_OK;
}

}  // namespace bnzi

extern "C" {

int bnz_diffuse(bnz_ctx* c, double dt, int* nsts_out) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (!(dt >= 0.)) return fail(c, BNZ_ERR_ARG, "dt must be >= 0");
  c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
  int rc = diffuse_impl(c, &c->d_ds->dt, dt, nsts_out);
  if (rc) return rc;
  if (c->md.path == BNZ_PATH_FUSED) {
    c->ghosts_stale = true;  // cons no longer matches prim
    rc = refresh_cds(c);
  }
  if (c->md.path == BNZ_PATH_SPLIT) c->cons_stale = true;
  return rc;
}

int bnz_vl2_step(bnz_ctx* c, double dt) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (!(dt >= 0.) || std::isinf(dt)) return fail(c, BNZ_ERR_ARG, "dt must be finite and >= 0");
  c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
  return step_impl(c, dt);
}

int bnz_advance(bnz_ctx* c, double tmax, int max_steps, double* time_out, long* step_out) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  int rc0 = sync_time(c);
  if (rc0) return rc0;
  int n = 0;
  while (c->time < tmax && (max_steps <= 0 || n < max_steps)) {
    double dt;
    if (!c->md.fixdt) {
      StepArgs a = step_args(c);
      c->launches += c->L->new_dt(a, c->prim, c->d_ds, c->md.cour, 0);
      DtState ds;
      CKC(cudaMemcpyAsync(&ds, c->d_ds, sizeof ds, cudaMemcpyDeviceToHost, c->stream));
      CKC(cudaStreamSynchronize(c->stream));
      dt = ds.dt;
      if (c->time + dt > tmax) dt = tmax - c->time;
    } else {
      dt = c->md.dt_fixed;
    }
    c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
    int rc = step_impl(c, dt);
    if (rc) return rc;
    c->time += dt;
    c->step += 1;
    c->last_dt = dt;
    ++n;
  }
  CKC(cudaStreamSynchronize(c->stream));
  if (time_out) *time_out = c->time;
  if (step_out) *step_out = c->step;
  return BNZ_OK;
}

int bnz_last_nsts(const bnz_ctx* c, int* nsts) {
  if (!c || !nsts) return BNZ_ERR_ARG;
  *nsts = c->last_nsts;
  return BNZ_OK;
}

int bnz_get_time(bnz_ctx* c, double* t, long* s, double* last_dt) {
  if (!c) return BNZ_ERR_ARG;
  int rc = sync_time(c);
  if (rc) return rc;
  if (t) *t = c->time;
  if (s) *s = c->step;
  if (last_dt) *last_dt = c->last_dt;
  return BNZ_OK;
}

int bnz_set_time(bnz_ctx* c, double t, long s) {
  if (!c) return BNZ_ERR_ARG;
  int rc = sync_time(c);
  if (rc) return rc;
  c->time = t;
  c->step = s;
  return BNZ_OK;
}

int bnz_check(bnz_ctx* c, uint32_t* bits) {
  if (!c || !c->d_err) return fail(c, BNZ_ERR_ARG, "context not created");
  unsigned h = 0;
  CKC(cudaMemcpyAsync(&h, c->d_err, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CKC(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  if (bits) *bits = h;
  if (h & 16u) return fail(c, BNZ_ERR_TIMEOUT, "a bounded device wait ran out");
  if (h) return fail(c, BNZ_ERR_STATE, "non-physical state on the device (error bits " + std::to_string(h) + ")");
  return BNZ_OK;
}

int bnz_sync(bnz_ctx* c) {
  if (!c || !c->stream) return fail(c, BNZ_ERR_ARG, "context not created");
  CKC(cudaStreamSynchronize(c->stream));
  return BNZ_OK;
}


int bnz_advance_graph(bnz_ctx* c, double tmax, int nsteps) {
  if (c && c->prim && drive_on(c->md)) {
    // new driving amplitudes every step come from the host: step without a graph
    double t;
    long st;
    return bnz_advance(c, tmax, nsteps, &t, &st);
  }
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (nsteps < 0) return fail(c, BNZ_ERR_ARG, "nsteps must be >= 0");
  if (c->md.kappa0 > 0.)
    return fail(c, BNZ_ERR_UNSUPPORTED, "graph stepping with conduction needs the host stage count");
  if (nsteps == 0) return BNZ_OK;
  // the fused path ping-pongs its state buffers, so a captured graph holds two
  // steps and returns the pointers to where they started
  const int unroll = c->md.path == BNZ_PATH_FUSED ? 2 : 1;
  if (!c->time_on_device) {
    // dt, time, tmax are the first three doubles of DtState; step follows cdsmax_bits
    double h[3] = {c->last_dt, c->time, tmax};
    long long st = c->step;
    c->h_stage[0] = h[0];
    c->h_stage[1] = h[1];
    c->h_stage[2] = h[2];
    c->h_step = st;
    CKC(cudaMemcpyAsync(c->d_ds, c->h_stage, 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CKC(cudaMemcpyAsync(&c->d_ds->step, &c->h_step, sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  } else {
    c->h_stage[2] = tmax;
    CKC(cudaMemcpyAsync(&c->d_ds->tmax, &c->h_stage[2], sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  auto one_step = [&](void) -> int {
    int rc;
    if (c->md.path == BNZ_PATH_FUSED) {
      rc = step_impl(c, 0., c->md.fixdt ? FDT_FIXED : FDT_CFL);
    } else {
      StepArgs a = step_args(c);
      if (!c->md.fixdt) c->launches += c->L->new_dt(a, c->prim, c->d_ds, c->md.cour, 1);
      else c->launches += c->L->fixed_dt(c->stream, c->d_ds, c->md.dt_fixed);
      rc = step_impl(c, 0.);
    }
    if (rc) return rc;
    c->launches += c->L->time_advance(c->stream, c->d_ds);
    return BNZ_OK;
  };
  int full = nsteps / unroll, rest = nsteps % unroll;
  if (full > 0) {
    if (c->graph && c->graph_parity != c->parity) {
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    if (!c->graph) {
      c->graph_parity = c->parity;
      CKC(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      long long before = c->launches;
      int rc = BNZ_OK;
      for (int u = 0; u < unroll && rc == BNZ_OK; ++u) rc = one_step();
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return fail(c, BNZ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&c->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(c, BNZ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
      c->graph_launches = c->launches - before;
      c->launches = before;
      // capture recorded the pointer swaps of `unroll` steps; replaying starts
      // from the parity it was captured at
      if (c->md.path == BNZ_PATH_FUSED) set_parity(c, c->graph_parity);
    }
    for (int r = 0; r < full; ++r) {
      CKC(cudaGraphLaunch(c->graph, c->stream));
      c->launches += c->graph_launches;
    }
    if (c->md.path == BNZ_PATH_FUSED) c->ghosts_stale = true;
    if (c->md.path == BNZ_PATH_SPLIT) c->cons_stale = true;
  }
  for (int r = 0; r < rest; ++r) {
    int rc = one_step();
    if (rc) return rc;
  }
  CKC(cudaGetLastError());
  c->time_on_device = true;
  return BNZ_OK;
}

int bnz_riemann(int rsolver, int nvar, const double* wl, const double* wr, const double* bx, double* flux, int n,
                double gam, int exact_fp, unsigned* err_bits, void* stream) {
  if (nvar != 6 && nvar != 9) return BNZ_ERR_ARG;
  if (!wl || !wr || !flux || (nvar == 9 && !bx) || n < 0 || !(gam > 1.)) return BNZ_ERR_ARG;
  if (rsolver < BNZ_RS_HLL || rsolver > BNZ_RS_HLLT) return BNZ_ERR_ARG;
  // hllc exists in the hydro build only, hlld in the MHD builds only
  if ((rsolver == BNZ_RS_HLLC && nvar != 6) || (rsolver == BNZ_RS_HLLD && nvar != 9)) return BNZ_ERR_UNSUPPORTED;
  // the hydro build's hllt is not built (its field-free star states differ)
  if (rsolver == BNZ_RS_HLLT && nvar != 9) return BNZ_ERR_UNSUPPORTED;
  if (n == 0) return BNZ_OK;
  const Launchers* L = exact_fp ? &exact::table : &fast::table;
  const int rs = (rsolver == BNZ_RS_HLL && nvar == 6) ? 4 : rsolver;  // 4: dev::RS_HLL_HYDRO
  L->riemann_rows(rs, wl, wr, bx, flux, n, nvar, gam, err_bits, (cudaStream_t)stream);
  return cudaGetLastError() == cudaSuccess ? BNZ_OK : BNZ_ERR_CUDA;
}

int bnz_device_state(bnz_ctx* c, double** prim, double** cons, double** bfld) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (prim) *prim = c->prim;
  if (cons) *cons = c->cons;
  if (bfld) *bfld = c->bfld;
  return BNZ_OK;
}

int bnz_set_stream(bnz_ctx* c, void* stream) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  CKC(cudaStreamSynchronize(c->stream));
  if (c->own_stream) cudaStreamDestroy(c->stream);
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  return BNZ_OK;
}

int bnz_launch_count(const bnz_ctx* c, long long* n) {
  if (!c) return BNZ_ERR_ARG;
  if (n) *n = c->launches;
  return BNZ_OK;
}

int bnz_stream(bnz_ctx* c, void** s) {
  if (!c) return BNZ_ERR_ARG;
  if (s) *s = (void*)c->stream;
  return BNZ_OK;
}

}  // extern "C"


// ===========================================================================
// Batches of independent grids (uneven parameter sweeps).  Every instance is a
// fused-path context on the batch's stream; one step of the whole batch is
// four launches (per-instance dt, predictor tiles, corrector tiles, time).
// ===========================================================================

struct bnz_batch {
  std::vector<bnz_ctx*> ctx;
  bnz_method_desc md;
  FusedInst* d_inst = nullptr;
  FusedTile* d_tiles = nullptr;
  int ntA = 0, ntB = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  cudaGraphExec_t graph = nullptr;
  int graph_parity = -1;
  int parity = 0;
  long long launches = 0;
  long long graph_launches = 0;
  double h_tmax = 0.;
  int variant = 0;
  const Launchers* L = nullptr;
  std::string err;
  // first predictor / corrector tile of every instance (n + 1 entries)
  std::vector<int> offA, offB;
  // host-state stepping: copy-in and copy-out streams and their events
  cudaStream_t cin = nullptr, cout = nullptr;
  std::vector<cudaEvent_t> hev;
  // persistent kernels: tensor maps of every instance's ws (corrector) and
  // w[0], w[1] (predictor), work-queue counters (corrector, predictor)
  unsigned char* d_maps = nullptr;
  unsigned char* d_wmaps = nullptr;
  unsigned* d_queue = nullptr;
  // host-state stepping through a device staging buffer laid out like
  // back-to-back host state (instance q: prim then bfld, at soff[q]), and the
  // segment tables between it and the instances' buffers of either parity
  int withhold = 0;  // test switch (bnz_batch_test_withhold_loads)
  double* d_stage = nullptr;
  std::vector<size_t> soff;
  struct SegCopy* d_segs[2] = {nullptr, nullptr};
  bool stage_failed = false;
  // 3D batches: instance records, chunk lists (predictor then corrector) and
  // the instances' 4D tensor maps of ws (128 bytes each)
  bool dims3 = false;
  bool split = false;  // 3D batch on the split path: each instance's step in turn
  FusedInst3* d_inst3 = nullptr;
  FusedTile3* d_tiles3 = nullptr;
  int ntA3 = 0, ntB3 = 0;
  unsigned char* d_maps3 = nullptr;
};

// One contiguous copy between the staging buffer (a) and an instance buffer (b).
struct SegCopy {
  double* a;
  double* b;
  long long n;
};

namespace {

int bfail(bnz_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

#define CKB(call)                                                                                \
  do {                                                                                           \
    cudaError_t _e = (call);                                                                     \
    if (_e != cudaSuccess)                                                                       \
      return bfail(b, BNZ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));        \
  } while (0)

FusedLaunch batch_launch(const bnz_batch* b, int dt_mode) {
  FusedLaunch f;
  memset(&f, 0, sizeof f);
  f.insts = b->d_inst;
  f.ninst = (int)b->ctx.size();
  f.tilesA = b->d_tiles;
  f.ntA = b->ntA;
  f.tilesB = b->d_tiles + b->ntA;
  f.ntB = b->ntB;
  f.rsolver = b->md.rsolver;
  f.limiter = b->md.limiter;
  f.charact_proj = b->md.charact_proj;
  f.variant = b->variant;
  f.cour = b->md.cour;
  f.dt_mode = dt_mode;
  f.dt_fixed = b->md.dt_fixed;
  f.err = b->ctx.empty() ? nullptr : b->ctx[0]->d_err;
  f.stream = b->stream;
  if (FUSED_VARIANTS[b->variant].persistent && b->d_maps) {
    f.wsmaps = b->d_maps;
    f.queue = b->d_queue;
    f.withhold = b->withhold;
    if (FUSED_VARIANTS[b->variant].persistent == 2) f.wmaps = b->d_wmaps;
  }
  return f;
}

Fused3Launch batch_launch3(const bnz_batch* b, int dt_mode) {
  Fused3Launch f;
  memset(&f, 0, sizeof f);
  f.insts = b->d_inst3;
  f.ninst = (int)b->ctx.size();
  f.tilesA = b->d_tiles3;
  f.ntA = b->ntA3;
  f.tilesB = b->d_tiles3 + b->ntA3;
  f.ntB = b->ntB3;
  f.rsolver = b->md.rsolver;
  f.limiter = b->md.limiter;
  f.charact_proj = b->md.charact_proj;
  f.cour = b->md.cour;
  f.dt_mode = dt_mode;
  f.dt_fixed = b->md.dt_fixed;
  f.wsmaps = b->d_maps3;
  f.stream = b->stream;
  return f;
}

// cuTensorMapEncodeTiled from the driver, found once through the runtime.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// A TMA box of (x, y, field) = (bw, bh, nf) doubles over one nf-field array of
// the instance (ws, w[p] or b[p]), bw even, used from even columns.  A map
// needs 16-byte row and field strides, so instances with odd Ntot_x get none
// (their tiles stage with plain loads).  Returns whether the map was made.
bool cell_map(const bnz_ctx* c, const double* base, int nf, int bw, int bh, CUtensorMap* out) {
  EncodeTiledFn enc = encode_tiled();
  const int nx = c->Ntot[0], ny = c->Ntot[1];
  if (!enc || (nx & 1) || ((uintptr_t)base & 15)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nf};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * sizeof(double), (cuuint64_t)nx * ny * sizeof(double)};
  const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, (cuuint32_t)nf};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)base, dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

namespace bnzi {
// A 4D map (x, y, z, field) over an nft-field array of a 3D context, with
// boxes of bx x by x bz cells and bf fields: the split kernels' TMA boxes.
// Needs even Ntot_x (16-byte strides).
bool split_map(const bnz_ctx* c, const double* base, int nft, int bx, int by, int bz, int bf, void* map128) {
  EncodeTiledFn enc = encode_tiled();
  const int nx = c->Ntot[0], ny = c->Ntot[1], nz = c->Ntot[2];
  if (!enc || (nx & 1) || ((uintptr_t)base & 15)) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nft};
  const cuuint64_t strides[3] = {(cuuint64_t)nx * sizeof(double), (cuuint64_t)nx * ny * sizeof(double),
                                 (cuuint64_t)nx * ny * nz * sizeof(double)};
  const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, (cuuint32_t)bf};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)base, dims, strides, box,
             es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The split kernels' maps into device memory, when every map can be made, in
// the order of split::TM_*: for the update (boxes of 34 x 9 cells, 1 or 2
// planes) prim, the three flux arrays, bfld, the b^n copy in ec, ee; for the
// corrector's PLM flux tiles, the predictor's prim in cons_s in the boxes of
// the x (34 x 8 x 1), y (16 x 18 x 1) and z (16 x 1 x 18) sweeps.
cudaError_t build_split_maps(bnz_ctx* c) {
  CUtensorMap m[10];
  const bool ok = split_map(c, c->prim, 9, 34, 9, 1, 9, &m[0]) && split_map(c, c->flx[0], 9, 34, 9, 1, 6, &m[1]) &&
                  split_map(c, c->flx[1], 9, 34, 9, 1, 6, &m[2]) && split_map(c, c->flx[2], 9, 34, 9, 2, 6, &m[3]) &&
                  split_map(c, c->bfld, 3, 34, 9, 2, 3, &m[4]) && split_map(c, c->ec, 3, 34, 9, 2, 3, &m[5]) &&
                  split_map(c, c->ee, 3, 34, 9, 2, 3, &m[6]) && split_map(c, c->cons_s, 9, 34, 8, 1, 9, &m[7]) &&
                  split_map(c, c->cons_s, 9, 16, 18, 1, 9, &m[8]) && split_map(c, c->cons_s, 9, 16, 1, 18, 9, &m[9]);
  if (!ok) return cudaSuccess;  // the kernel without TMA runs
  cudaError_t e = cudaMalloc((void**)&c->d_smaps, sizeof m);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_smaps, m, sizeof m, cudaMemcpyHostToDevice);
  return e;
}

bool ws_map3(const bnz_ctx* c, const double* base, void* map128) {
  EncodeTiledFn enc = encode_tiled();
  const int nx = c->Ntot[0], ny = c->Ntot[1], nz = c->Ntot[2];
  if (!enc || (nx & 1) || ((uintptr_t)base & 15)) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, 9};
  const cuuint64_t strides[3] = {(cuuint64_t)nx * sizeof(double), (cuuint64_t)nx * ny * sizeof(double),
                                 (cuuint64_t)nx * ny * nz * sizeof(double)};
  const cuuint32_t box[4] = {(cuuint32_t)F3_BW, (cuuint32_t)F3_BH, 1, 9};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)base, dims, strides, box,
             es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace bnzi

namespace {

// Tile lists of every instance for the batch's variant (predictor list first).
int batch_build_tiles(bnz_batch* b) {
  const FusedVariant& v = FUSED_VARIANTS[b->variant];
  std::vector<FusedTile> tA, tB;
  b->offA.assign(1, 0);
  b->offB.assign(1, 0);
  for (int q = 0; q < (int)b->ctx.size(); ++q) {
    const bnz_ctx* c = b->ctx[q];
    if (v.persistent == 2) make_tiles_uniform(q, c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->ng, v.tx, v.ty, tA);
    else make_tiles(q, c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->ng, true, v.tx, v.ty, tA);
    make_tiles(q, c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->ng, false, v.tx, v.ty, tB);
    b->offA.push_back((int)tA.size());
    b->offB.push_back((int)tB.size());
  }
  if (v.persistent) {
    static_assert(sizeof(CUtensorMap) == 128, "tensor maps are 128 bytes");
    // 6 maps per instance (TmaBox<tx, ty> in bnz_fused.cuh): ws with tx + 4
    // cells from an even column and ty + 4 rows; w[0], w[1] (9 fields) and
    // b[0], b[1] (3 faces) with tx + 1 positions from an even column and ty + 1
    // rows; bs (its first 2 fields, an L2 prefetch box) with tx + 2 positions
    // and ty + 2 rows
    const int bw = (v.tx + 6) & ~1, bh = v.ty + 4;
    const int cw = (v.tx + 3) & ~1, ch = v.ty + 1;
    const int pw = (v.tx + 4) & ~1, ph = v.ty + 2;
    std::vector<CUtensorMap> maps(6 * b->ctx.size());
    std::vector<int> ok(b->ctx.size(), 0);
    memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    for (size_t q = 0; q < b->ctx.size(); ++q) {
      const bnz_ctx* c = b->ctx[q];
      CUtensorMap* m = &maps[6 * q];
      ok[q] = cell_map(c, c->cons_s, 9, bw, bh, &m[0]) && cell_map(c, c->wbuf[0], 9, cw, ch, &m[1]) &&
              cell_map(c, c->wbuf[1], 9, cw, ch, &m[2]) && cell_map(c, c->bbuf[0], 3, cw, ch, &m[3]) &&
              cell_map(c, c->bbuf[1], 3, cw, ch, &m[4]) && cell_map(c, c->bfld_s, 2, pw, ph, &m[5]);
    }
    for (FusedTile& t : tB) t.tma = ok[t.inst];
    if (!b->d_maps) CKB(cudaMalloc((void**)&b->d_maps, maps.size() * sizeof(CUtensorMap)));
    if (!b->d_queue) CKB(cudaMalloc((void**)&b->d_queue, 2 * sizeof(unsigned)));
    CKB(cudaMemcpy(b->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    CKB(cudaMemset(b->d_queue, 0, 2 * sizeof(unsigned)));
  }
  if (v.persistent == 2) {
    // predictor: boxes of TmaBoxP<tx, ty> over w[0], w[1] (9 fields) and
    // b[0], b[1] (3 faces): tx + 2 cells from an even column, ty + 2 rows;
    // only full interior tiles use them
    const int bw = (v.tx + 4) & ~1, bh = v.ty + 2;
    std::vector<CUtensorMap> maps(4 * b->ctx.size());
    std::vector<int> ok(b->ctx.size(), 0);
    memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    for (size_t q = 0; q < b->ctx.size(); ++q) {
      const bnz_ctx* c = b->ctx[q];
      ok[q] = cell_map(c, c->wbuf[0], 9, bw, bh, &maps[4 * q]) && cell_map(c, c->wbuf[1], 9, bw, bh, &maps[4 * q + 1]) &&
              cell_map(c, c->bbuf[0], 3, bw, bh, &maps[4 * q + 2]) && cell_map(c, c->bbuf[1], 3, bw, bh, &maps[4 * q + 3]);
    }
    for (FusedTile& t : tA) {
      const bnz_ctx* c = b->ctx[t.inst];
      const int ng = c->ng, n0 = c->i2 - c->i1 + 1, n1 = c->j2 - c->j1 + 1;
      const bool interior = t.x0 - 1 >= ng && t.x0 + t.wx <= ng + n0 - 1 && t.y0 - 1 >= ng &&
                            t.y0 + t.wy <= ng + n1 - 1;
      t.tma = !ok[t.inst] ? 0 : (interior && t.wx == v.tx && t.wy == v.ty) ? 1 : 2;
    }
    if (!b->d_wmaps) CKB(cudaMalloc((void**)&b->d_wmaps, maps.size() * sizeof(CUtensorMap)));
    CKB(cudaMemcpy(b->d_wmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  }
  b->ntA = (int)tA.size();
  b->ntB = (int)tB.size();
  tA.insert(tA.end(), tB.begin(), tB.end());
  if (b->d_tiles) cudaFree(b->d_tiles);
  b->d_tiles = nullptr;
  CKB(cudaMalloc((void**)&b->d_tiles, tA.size() * sizeof(FusedTile)));
  CKB(cudaMemcpy(b->d_tiles, tA.data(), tA.size() * sizeof(FusedTile), cudaMemcpyHostToDevice));
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return BNZ_OK;
}

// Instance records, chunk lists and tensor maps of a 3D batch: every
// instance's chunks in one predictor list and one corrector list.
int batch_build3(bnz_batch* b) {
  const int n = (int)b->ctx.size();
  std::vector<FusedInst3> insts;
  std::vector<FusedTile3> tA, tB;
  std::vector<CUtensorMap> maps(n);
  memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  for (int q = 0; q < n; ++q) {
    const bnz_ctx* c = b->ctx[q];
    insts.push_back(make_inst3(c));
    const int N[3] = {c->i2 - c->i1 + 1, c->j2 - c->j1 + 1, c->k2 - c->k1 + 1};
    make_tiles3(q, N, c->ng, true, F3_TX, F3_TY, F3_KZ, tA);
    const size_t b0 = tB.size();
    make_tiles3(q, N, c->ng, false, F3_TX, F3_TY, F3_KZ, tB);
    const bool ok = ws_map3(c, c->cons_s, &maps[q]);
    for (size_t t = b0; t < tB.size(); ++t) tB[t].tma = ok ? 1 : 0;
  }
  b->ntA3 = (int)tA.size();
  b->ntB3 = (int)tB.size();
  tA.insert(tA.end(), tB.begin(), tB.end());
  CKB(cudaMalloc((void**)&b->d_inst3, insts.size() * sizeof(FusedInst3)));
  CKB(cudaMemcpy(b->d_inst3, insts.data(), insts.size() * sizeof(FusedInst3), cudaMemcpyHostToDevice));
  CKB(cudaMalloc((void**)&b->d_tiles3, tA.size() * sizeof(FusedTile3)));
  CKB(cudaMemcpy(b->d_tiles3, tA.data(), tA.size() * sizeof(FusedTile3), cudaMemcpyHostToDevice));
  CKB(cudaMalloc((void**)&b->d_maps3, maps.size() * sizeof(CUtensorMap)));
  CKB(cudaMemcpy(b->d_maps3, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  return BNZ_OK;
}

template <class IT>
__global__ void k_set_tmax(IT* insts, int n, double tmax) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) insts[q].ds->tmax = tmax;
}

// Copies of the segments segs[0 .. gridDim.y-1]: staging -> instance when
// to_instance, else instance -> staging.
// 16-byte copies where both ends are 16-byte aligned (the staging offsets are
// multiples of 12 doubles, the instance buffers are allocation starts).
__global__ void k_segcopy(const SegCopy* __restrict__ segs, int to_instance) {
  const SegCopy sg = segs[blockIdx.y];
  const double* __restrict__ src = to_instance ? sg.a : sg.b;
  double* __restrict__ dst = to_instance ? sg.b : sg.a;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if ((((uintptr_t)src | (uintptr_t)dst) & 15) == 0) {
    const long long n2 = sg.n >> 1;
    const double2* __restrict__ s2 = reinterpret_cast<const double2*>(src);
    double2* __restrict__ d2 = reinterpret_cast<double2*>(dst);
    for (long long i = i0; i < n2; i += stride) d2[i] = s2[i];
    if ((sg.n & 1) && i0 == 0) dst[sg.n - 1] = src[sg.n - 1];
  } else {
    for (long long i = i0; i < sg.n; i += stride) dst[i] = src[i];
  }
}

// Clears the CFL slot `parity` of instances q0 .. q0+n-1 before k_cds_batch
// folds the maximum of a freshly loaded state into it.
__global__ void k_cds_clear(FusedInst* insts, int q0, int n, int parity) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) insts[q0 + q].ds->cds_bits[parity] = 0ULL;
}

}  // namespace

extern "C" {

int bnz_batch_create(const bnz_grid_desc* grids, int n, const bnz_method_desc* md, bnz_batch** out) {
  if (!grids || !md || !out || n < 1) return BNZ_ERR_ARG;
  bnz_batch* b = new bnz_batch();
  *out = b;
  b->md = *md;
  b->dims3 = grids[0].dims == 3;
  for (int q = 0; q < n; ++q)
    if (grids[q].dims != grids[0].dims || (grids[q].dims != 2 && grids[q].dims != 3))
      return bfail(b, BNZ_ERR_UNSUPPORTED, "a batch takes 2D grids or 3D grids, not a mix");
  // 3D batches run the fused chunk kernels over every instance in one launch
  // per stage, or (path = split) the split path's launches instance by
  // instance; 2D batches run the fused tile kernels
  b->split = md->path == BNZ_PATH_SPLIT;
  if (b->split && !b->dims3)
    return bfail(b, BNZ_ERR_UNSUPPORTED, "the split path batches 3D grids (2D batches run the fused tile kernels)");
  b->md.path = b->split ? BNZ_PATH_SPLIT : BNZ_PATH_FUSED;
  if (md->kappa0 > 0. && !b->dims3)
    return bfail(b, BNZ_ERR_UNSUPPORTED, "2D batches advance the hyperbolic step only (kappa0 = 0)");
  if (drive_on(*md)) return bfail(b, BNZ_ERR_UNSUPPORTED, "batches do not drive turbulence (drive_f0 = 0)");
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bfail(b, BNZ_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  std::vector<FusedInst> insts;
  for (int q = 0; q < n; ++q) {
    bnz_ctx* c = nullptr;
    int rc = bnz_create(&grids[q], &b->md, &c);
    if (rc) {
      std::string m = "instance " + std::to_string(q) + ": " + (c ? c->err : std::string("create failed"));
      if (c) bnz_destroy(c);
      return bfail(b, rc, m);
    }
    b->ctx.push_back(c);
    rc = bnz_set_stream(c, (void*)b->stream);
    if (rc) return bfail(b, rc, c->err);
    if (!b->split) insts.push_back(make_inst(c));
  }
  b->L = b->ctx[0]->L;
  if (b->split) return BNZ_OK;
  if (b->dims3) {
    b->variant = 0;
    return batch_build3(b);
  }
  CKB(cudaMalloc((void**)&b->d_inst, insts.size() * sizeof(FusedInst)));
  CKB(cudaMemcpy(b->d_inst, insts.data(), insts.size() * sizeof(FusedInst), cudaMemcpyHostToDevice));
  b->variant = BATCH_DEFAULT_VARIANT;
  return batch_build_tiles(b);
}

int bnz_batch_destroy(bnz_batch* b) {
  if (!b) return BNZ_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (bnz_ctx* c : b->ctx) bnz_destroy(c);
  if (b->d_inst) cudaFree(b->d_inst);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_maps) cudaFree(b->d_maps);
  if (b->d_wmaps) cudaFree(b->d_wmaps);
  if (b->d_stage) cudaFree(b->d_stage);
  for (SegCopy* sg : b->d_segs)
    if (sg) cudaFree(sg);
  if (b->d_queue) cudaFree(b->d_queue);
  if (b->d_inst3) cudaFree(b->d_inst3);
  if (b->d_tiles3) cudaFree(b->d_tiles3);
  if (b->d_maps3) cudaFree(b->d_maps3);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->cin) cudaStreamSynchronize(b->cin);
  if (b->cout) cudaStreamSynchronize(b->cout);
  for (cudaEvent_t e : b->hev) cudaEventDestroy(e);
  if (b->cin) cudaStreamDestroy(b->cin);
  if (b->cout) cudaStreamDestroy(b->cout);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return BNZ_OK;
}

const char* bnz_batch_last_error(const bnz_batch* b) { return b ? b->err.c_str() : "null batch"; }

int bnz_batch_size(const bnz_batch* b, int* n) {
  if (!b) return BNZ_ERR_ARG;
  if (n) *n = (int)b->ctx.size();
  return BNZ_OK;
}

int bnz_batch_instance(bnz_batch* b, int i, bnz_ctx** ctx) {
  if (!b || i < 0 || i >= (int)b->ctx.size() || !ctx) return bfail(b, BNZ_ERR_ARG, "instance index out of range");
  *ctx = b->ctx[i];
  return BNZ_OK;
}

int bnz_batch_set_stream(bnz_batch* b, void* stream) {
  if (!b) return BNZ_ERR_ARG;
  CKB(cudaStreamSynchronize(b->stream));
  // move the instances first: they still reference the old stream
  for (bnz_ctx* c : b->ctx) {
    int rc = bnz_set_stream(c, stream);
    if (rc) return bfail(b, rc, c->err);
  }
  if (b->own_stream) cudaStreamDestroy(b->stream);
  b->stream = (cudaStream_t)stream;
  b->own_stream = false;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return BNZ_OK;
}

}  // extern "C"

namespace {

// Common start of a batch advance: every instance must be at the batch parity
// with its time record on the device; then the stop time is set.
int batch_prologue(bnz_batch* b, double tmax) {
  for (bnz_ctx* c : b->ctx) {
    if (c->parity != b->parity) return bfail(b, BNZ_ERR_STATE, "instance stepped outside the batch");
    if (!c->time_on_device) {
      c->h_stage[0] = c->last_dt;
      c->h_stage[1] = c->time;
      c->h_stage[2] = tmax;
      c->h_step = c->step;
      CKB(cudaMemcpyAsync(c->d_ds, c->h_stage, 3 * sizeof(double), cudaMemcpyHostToDevice, b->stream));
      CKB(cudaMemcpyAsync(&c->d_ds->step, &c->h_step, sizeof(long long), cudaMemcpyHostToDevice, b->stream));
      c->time_on_device = true;
    }
  }
  const int n = (int)b->ctx.size();
  if (b->split) {
    for (bnz_ctx* c : b->ctx) {
      c->h_stage[2] = tmax;
      CKB(cudaMemcpyAsync(&c->d_ds->tmax, &c->h_stage[2], sizeof(double), cudaMemcpyHostToDevice, b->stream));
    }
    return BNZ_OK;
  }
  if (b->dims3) k_set_tmax<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_inst3, n, tmax);
  else k_set_tmax<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_inst, n, tmax);
  b->launches += 1;
  return BNZ_OK;
}

// One step of a 3D batch with conduction: the hyperbolic step of every
// instance in one launch per stage, then each instance's RKL2 conduction over
// its own dt (vanleer.pyx:147-151; the stage count is chosen on the host from
// the instance's dt, read back after the step).
int batch_step3_diffuse(bnz_batch* b) {
  const int mode = b->md.fixdt ? FDT_FIXED : FDT_CFL;
  const Fused3Launch f = batch_launch3(b, mode);
  b->launches += b->L->fused3_step(f, b->parity);
  const int n = (int)b->ctx.size();
  std::vector<DtState> ds(n);
  for (int q = 0; q < n; ++q)
    CKB(cudaMemcpyAsync(&ds[q], b->ctx[q]->d_ds, sizeof(DtState), cudaMemcpyDeviceToHost, b->stream));
  CKB(cudaStreamSynchronize(b->stream));
  b->parity ^= 1;
  for (int q = 0; q < n; ++q) {
    bnz_ctx* c = b->ctx[q];
    set_parity(c, b->parity);
    c->ghosts_stale = true;
    if (ds[q].dt > 0.) {
      int rc = diffuse_impl(c, &c->d_ds->dt, ds[q].dt, nullptr);
      if (!rc) rc = refresh_cds(c);
      if (rc) return bfail(b, rc, c->err);
    }
  }
  b->launches += b->L->fused3_time(f);
  return BNZ_OK;
}

void batch_epilogue(bnz_batch* b) {
  for (bnz_ctx* c : b->ctx) {
    if (b->split) {
      c->cons_stale = true;
    } else {
      set_parity(c, b->parity);
      c->ghosts_stale = true;
    }
    c->time_on_device = true;
  }
}

// One step of every instance of a split batch, in turn: the device CFL dt
// clipped to the instance's tmax, the split step and its boundary fill, the
// time record.  With conduction the stage count of each instance's RKL2 comes
// from its dt on the host (one read-back of every instance's dt per step); an
// instance at its tmax is not stepped.  An instance whose dt is zero on the
// graph path passes through the step unchanged (the update kernels return
// when dt is zero).
int batch_step_split(bnz_batch* b, bool host_dt) {
  const int n = (int)b->ctx.size();
  for (bnz_ctx* c : b->ctx) {
    StepArgs a = step_args(c);
    if (!c->md.fixdt) c->launches += c->L->new_dt(a, c->prim, c->d_ds, c->md.cour, 1);
    else c->launches += c->L->fixed_dt(c->stream, c->d_ds, c->md.dt_fixed);
  }
  std::vector<DtState> ds(host_dt ? n : 0);
  if (host_dt) {
    for (int q = 0; q < n; ++q)
      CKB(cudaMemcpyAsync(&ds[q], b->ctx[q]->d_ds, sizeof(DtState), cudaMemcpyDeviceToHost, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
  }
  for (int q = 0; q < n; ++q) {
    bnz_ctx* c = b->ctx[q];
    if (host_dt && !(ds[q].dt > 0.)) continue;
    int rc = step_impl(c, host_dt ? ds[q].dt : 0.);
    if (rc) return bfail(b, rc, c->err);
    c->launches += c->L->time_advance(c->stream, c->d_ds);
  }
  return BNZ_OK;
}

}  // namespace

extern "C" {

int bnz_batch_advance(bnz_batch* b, double tmax, int nsteps) {
  if (!b || b->ctx.empty()) return BNZ_ERR_ARG;
  if (nsteps < 0) return bfail(b, BNZ_ERR_ARG, "nsteps must be >= 0");
  if (nsteps == 0) return BNZ_OK;
  int rc = batch_prologue(b, tmax);
  if (rc) return rc;
  const int mode = b->md.fixdt ? FDT_FIXED : FDT_CFL;
  if (b->split) {
    const bool host_dt = b->md.kappa0 > 0.;
    if (host_dt) {
      // conduction's stage count is chosen on the host: no graph
      for (int s = 0; s < nsteps && rc == BNZ_OK; ++s) rc = batch_step_split(b, true);
    } else {
      if (!b->graph) {
        long long before = 0;
        for (const bnz_ctx* c : b->ctx) before += c->launches;
        CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = batch_step_split(b, false);
        // the captured launches run at each replay, not at capture
        long long after = 0;
        for (const bnz_ctx* c : b->ctx) after += c->launches;
        b->graph_launches = after - before;
        b->launches -= b->graph_launches;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
          if (g) cudaGraphDestroy(g);
          return rc;
        }
        if (e != cudaSuccess) return bfail(b, BNZ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, BNZ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
      }
      for (int s = 0; s < nsteps; ++s) {
        CKB(cudaGraphLaunch(b->graph, b->stream));
        b->launches += b->graph_launches;
      }
    }
    if (rc) return rc;
    CKB(cudaGetLastError());
    batch_epilogue(b);
    return BNZ_OK;
  }
  if (b->dims3 && b->md.kappa0 > 0.) {
    // conduction's stage count is chosen on the host: no graph
    for (int s = 0; s < nsteps; ++s) {
      rc = batch_step3_diffuse(b);
      if (rc) return rc;
    }
    CKB(cudaGetLastError());
    batch_epilogue(b);
    return BNZ_OK;
  }
  auto one_step = [&](int p) {
    if (b->dims3) {
      const Fused3Launch f = batch_launch3(b, mode);
      b->launches += b->L->fused3_step(f, p);
      b->launches += b->L->fused3_time(f);
      return;
    }
    FusedLaunch f = batch_launch(b, mode);
    b->launches += b->L->fused_step(f, p);
    b->launches += b->L->fused_time(f);
  };
  int full = nsteps / 2, rest = nsteps % 2;
  if (full > 0) {
    if (b->graph && b->graph_parity != b->parity) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    if (!b->graph) {
      b->graph_parity = b->parity;
      CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      long long before = b->launches;
      one_step(b->parity);
      one_step(b->parity ^ 1);
      cudaGraph_t g = nullptr;
      CKB(cudaStreamEndCapture(b->stream, &g));
      cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return bfail(b, BNZ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
      b->graph_launches = b->launches - before;
      b->launches = before;
    }
    for (int r = 0; r < full; ++r) {
      CKB(cudaGraphLaunch(b->graph, b->stream));
      b->launches += b->graph_launches;
    }
  }
  if (rest) {
    one_step(b->parity);
    b->parity ^= 1;
  }
  CKB(cudaGetLastError());
  batch_epilogue(b);
  return BNZ_OK;
}

int bnz_batch_advance_timed(bnz_batch* b, double tmax, int nsteps, double* ms_kernels) {
  if (!b || b->ctx.empty() || !ms_kernels) return BNZ_ERR_ARG;
  if (nsteps < 1) return bfail(b, BNZ_ERR_ARG, "nsteps must be >= 1");
  int rc = batch_prologue(b, tmax);
  if (rc) return rc;
  const int mode = b->md.fixdt ? FDT_FIXED : FDT_CFL;
  // one event set per step, so every launch of the run is timed
  std::vector<cudaEvent_t> ev(4 * (size_t)nsteps, nullptr);
  for (auto& e : ev) CKB(cudaEventCreate(&e));
  if ((b->dims3 && b->md.kappa0 > 0.) || b->split) {
    for (auto& x : ev) cudaEventDestroy(x);
    return bfail(b, BNZ_ERR_UNSUPPORTED, "per-launch timing covers fused batches without conduction");
  }
  for (int s = 0; s < nsteps; ++s) {
    if (b->dims3) {
      Fused3Launch f = batch_launch3(b, mode);
      f.events = &ev[4 * (size_t)s];
      b->launches += b->L->fused3_step(f, b->parity);
      b->launches += b->L->fused3_time(f);
    } else {
      FusedLaunch f = batch_launch(b, mode);
      f.events = &ev[4 * (size_t)s];
      b->launches += b->L->fused_step(f, b->parity);
      b->launches += b->L->fused_time(f);
    }
    b->parity ^= 1;
  }
  CKB(cudaGetLastError());
  cudaError_t e = cudaEventSynchronize(ev.back());
  double sum[3] = {0., 0., 0.};
  for (int s = 0; s < nsteps && e == cudaSuccess; ++s)
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
      float t = 0.f;
      e = cudaEventElapsedTime(&t, ev[4 * (size_t)s + k], ev[4 * (size_t)s + k + 1]);
      sum[k] += t;
    }
  for (auto& x : ev) cudaEventDestroy(x);
  if (e != cudaSuccess) return bfail(b, BNZ_ERR_CUDA, std::string("kernel timing: ") + cudaGetErrorString(e));
  for (int k = 0; k < 3; ++k) ms_kernels[k] = sum[k] / nsteps;
  batch_epilogue(b);
  return BNZ_OK;
}

}  // extern "C"

namespace {

// The staging buffer and segment tables, made on first use.  Without device
// memory for them the host copies go to the instances' buffers one by one.
bool stage_ready(bnz_batch* b) {
  if (b->d_stage) return true;
  if (b->stage_failed) return false;
  const int n = (int)b->ctx.size();
  b->soff.assign(n + 1, 0);
  for (int q = 0; q < n; ++q) b->soff[q + 1] = b->soff[q] + 12 * b->ctx[q]->ncell;
  if (cudaMalloc((void**)&b->d_stage, b->soff[n] * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    b->d_stage = nullptr;
    b->stage_failed = true;
    return false;
  }
  for (int p = 0; p < 2; ++p) {
    std::vector<SegCopy> segs(2 * n);
    for (int q = 0; q < n; ++q) {
      const bnz_ctx* c = b->ctx[q];
      segs[2 * q] = SegCopy{b->d_stage + b->soff[q], c->wbuf[p], 9 * (long long)c->ncell};
      segs[2 * q + 1] = SegCopy{b->d_stage + b->soff[q] + 9 * c->ncell, c->bbuf[p], 3 * (long long)c->ncell};
    }
    if (cudaMalloc((void**)&b->d_segs[p], segs.size() * sizeof(SegCopy)) != cudaSuccess ||
        cudaMemcpy(b->d_segs[p], segs.data(), segs.size() * sizeof(SegCopy), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
      cudaGetLastError();
      cudaFree(b->d_stage);
      b->d_stage = nullptr;
      b->stage_failed = true;
      return false;
    }
  }
  return true;
}

// Host <-> staging copies of instances q0 .. q1-1: one copy per run of host
// memory laid out like the staging buffer (prim[q], then bfld[q], then
// prim[q+1], ...), two per instance otherwise.
int stage_copies(bnz_batch* b, double* const* prim, double* const* bfld, int q0, int q1, bool in) {
  cudaStream_t st = in ? b->cin : b->cout;
  const cudaMemcpyKind kind = in ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  auto copy = [&](double* host, size_t off, size_t count) {
    double* dev = b->d_stage + off;
    return in ? cudaMemcpyAsync(dev, host, count * sizeof(double), kind, st)
              : cudaMemcpyAsync(host, dev, count * sizeof(double), kind, st);
  };
  int q = q0;
  while (q < q1) {
    const size_t nc = b->ctx[q]->ncell;
    if (bfld[q] != prim[q] + 9 * nc) {
      CKB(copy(prim[q], b->soff[q], 9 * nc));
      CKB(copy(bfld[q], b->soff[q] + 9 * nc, 3 * nc));
      ++q;
      continue;
    }
    int e = q + 1;  // run of self-contiguous instances that follow one another
    while (e < q1 && prim[e] == bfld[e - 1] + 3 * b->ctx[e - 1]->ncell &&
           bfld[e] == prim[e] + 9 * b->ctx[e]->ncell)
      ++e;
    CKB(copy(prim[q], b->soff[q], b->soff[e] - b->soff[q]));
    q = e;
  }
  return BNZ_OK;
}

}  // namespace

extern "C" {

int bnz_batch_step_host(bnz_batch* b, double* const* prim, double* const* bfld, double tmax, int nsteps,
                        int nchunks) {
  if (!b || b->ctx.empty()) return BNZ_ERR_ARG;
  const int n = (int)b->ctx.size();
  if (!prim || !bfld) return bfail(b, BNZ_ERR_ARG, "null host state arrays");
  for (int q = 0; q < n; ++q)
    if (!prim[q] || !bfld[q]) return bfail(b, BNZ_ERR_ARG, "null host state of instance " + std::to_string(q));
  if (nsteps < 1) return bfail(b, BNZ_ERR_ARG, "nsteps must be >= 1");
  if (b->dims3) return bfail(b, BNZ_ERR_UNSUPPORTED, "host-state stepping covers 2D batches");
  if (nchunks <= 0) nchunks = 32;
  if (nchunks > n) nchunks = n;
  int rc = batch_prologue(b, tmax);
  if (rc) return rc;
  if (!b->cin) {
    CKB(cudaStreamCreateWithFlags(&b->cin, cudaStreamNonBlocking));
    CKB(cudaStreamCreateWithFlags(&b->cout, cudaStreamNonBlocking));
  }
  while ((int)b->hev.size() < 2 * nchunks + 2) {
    cudaEvent_t e = nullptr;
    CKB(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->hev.push_back(e);
  }
  cudaEvent_t ev_entry = b->hev[0], ev_out = b->hev[1];
  // chunks of consecutive instances holding about equal numbers of cells
  std::vector<int> cut(1, 0);
  {
    double total = 0., acc = 0.;
    for (bnz_ctx* c : b->ctx) total += (double)c->ncell;
    for (int q = 0; q < n; ++q) {
      acc += (double)b->ctx[q]->ncell;
      const int left = n - (q + 1);
      const int want = (int)cut.size();  // index of the chunk being closed
      if (want < nchunks && acc >= total * want / nchunks && left >= nchunks - want) cut.push_back(q + 1);
    }
    if (cut.back() != n) cut.push_back(n);
  }
  const int nc = (int)cut.size() - 1;
  const bool staged = stage_ready(b);
  // the copies in follow whatever the compute stream holds already
  CKB(cudaEventRecord(ev_entry, b->stream));
  CKB(cudaStreamWaitEvent(b->cin, ev_entry, 0));
  for (int k = 0; k < nc; ++k) {
    if (staged) {
      rc = stage_copies(b, prim, bfld, cut[k], cut[k + 1], true);
      if (rc) return rc;
    } else {
      for (int q = cut[k]; q < cut[k + 1]; ++q) {
        bnz_ctx* c = b->ctx[q];
        CKB(cudaMemcpyAsync(c->prim, prim[q], 9 * c->ncell * sizeof(double), cudaMemcpyHostToDevice, b->cin));
        CKB(cudaMemcpyAsync(c->bfld, bfld[q], 3 * c->ncell * sizeof(double), cudaMemcpyHostToDevice, b->cin));
      }
    }
    CKB(cudaEventRecord(b->hev[2 + 2 * k], b->cin));
  }
  const int mode = b->md.fixdt ? FDT_FIXED : FDT_CFL;
  const int p0 = b->parity, p1 = (p0 + nsteps) & 1;
  for (int k = 0; k < nc; ++k) {
    const int q0 = cut[k], q1 = cut[k + 1];
    FusedLaunch f = batch_launch(b, mode);
    f.inst0 = q0;
    f.ninst = q1 - q0;
    f.tilesA = b->d_tiles + b->offA[q0];
    f.ntA = b->offA[q1] - b->offA[q0];
    f.tilesB = b->d_tiles + b->ntA + b->offB[q0];
    f.ntB = b->offB[q1] - b->offB[q0];
    CKB(cudaStreamWaitEvent(b->stream, b->hev[2 + 2 * k], 0));
    if (staged) {
      // staging buffer -> the instances' buffers of the current parity
      k_segcopy<<<dim3(128, 2 * (q1 - q0)), 256, 0, b->stream>>>(b->d_segs[p0] + 2 * q0, 1);
      b->launches += 1;
    }
    // the loaded state's CFL maximum, then the steps
    k_cds_clear<<<(f.ninst + 127) / 128, 128, 0, b->stream>>>(b->d_inst, q0, f.ninst, p0);
    b->launches += 1 + b->L->fused_cds(f, p0);
    int p = p0;
    for (int s = 0; s < nsteps; ++s) {
      b->launches += b->L->fused_step(f, p);
      b->launches += b->L->fused_time(f);
      p ^= 1;
    }
    // ghosts of the result, as bnz_get_state returns them
    for (int q = q0; q < q1; ++q) {
      bnz_ctx* c = b->ctx[q];
      set_parity(c, p1);
      StepArgs a = step_args(c);
      b->launches += c->L->apply_bc(a, c->prim, c->bfld, 0xFFFu);
    }
    if (staged) {
      // the results -> staging buffer (its part for this group was consumed above)
      k_segcopy<<<dim3(128, 2 * (q1 - q0)), 256, 0, b->stream>>>(b->d_segs[p1] + 2 * q0, 0);
      b->launches += 1;
    }
    CKB(cudaEventRecord(b->hev[3 + 2 * k], b->stream));
    CKB(cudaStreamWaitEvent(b->cout, b->hev[3 + 2 * k], 0));
    if (staged) {
      rc = stage_copies(b, prim, bfld, q0, q1, false);
      if (rc) return rc;
    } else {
      for (int q = q0; q < q1; ++q) {
        bnz_ctx* c = b->ctx[q];
        CKB(cudaMemcpyAsync(prim[q], c->prim, 9 * c->ncell * sizeof(double), cudaMemcpyDeviceToHost, b->cout));
        CKB(cudaMemcpyAsync(bfld[q], c->bfld, 3 * c->ncell * sizeof(double), cudaMemcpyDeviceToHost, b->cout));
      }
    }
  }
  CKB(cudaGetLastError());
  CKB(cudaEventRecord(ev_out, b->cout));
  CKB(cudaStreamWaitEvent(b->stream, ev_out, 0));
  b->parity = p1;
  batch_epilogue(b);  // cons is not derived here: ghosts stay marked stale
  CKB(cudaStreamSynchronize(b->stream));
  return BNZ_OK;
}

int bnz_batch_test_withhold_loads(bnz_batch* b, int on) {
  if (!b) return BNZ_ERR_ARG;
  CKB(cudaStreamSynchronize(b->stream));
  b->withhold = on ? 1 : 0;
  if (b->graph) {  // a captured step holds the old value
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return BNZ_OK;
}

int bnz_batch_launch_count(const bnz_batch* b, long long* n) {
  if (!b) return BNZ_ERR_ARG;
  long long t = b->launches;
  for (const bnz_ctx* c : b->ctx) t += c->launches;
  if (n) *n = t;
  return BNZ_OK;
}

int bnz_batch_sync(bnz_batch* b) {
  if (!b) return BNZ_ERR_ARG;
  CKB(cudaStreamSynchronize(b->stream));
  return BNZ_OK;
}

int bnz_variant_count(int* n, int* tx, int* ty, int* staged, int* persistent) {
  if (n) *n = FUSED_NVARIANT;
  for (int v = 0; v < FUSED_NVARIANT; ++v) {
    if (tx) tx[v] = FUSED_VARIANTS[v].tx;
    if (ty) ty[v] = FUSED_VARIANTS[v].ty;
    if (staged) staged[v] = FUSED_VARIANTS[v].staged;
    if (persistent) persistent[v] = FUSED_VARIANTS[v].persistent;
  }
  return BNZ_OK;
}

int bnz_batch_set_variant(bnz_batch* b, int v) {
  if (!b) return BNZ_ERR_ARG;
  if (b->dims3) return v == 0 ? BNZ_OK : bfail(b, BNZ_ERR_UNSUPPORTED, "3D batches have one kernel shape");
  if (v < 0 || v >= FUSED_NVARIANT) return bfail(b, BNZ_ERR_ARG, "variant out of range");
  if (!fused_variant_built(v, b->md.rsolver == BNZ_RS_HLLD))
    return bfail(b, BNZ_ERR_UNSUPPORTED, "variants 1-7 are built for hlld only");
  if (v == b->variant) return BNZ_OK;
  CKB(cudaStreamSynchronize(b->stream));
  b->variant = v;
  return batch_build_tiles(b);
}

int bnz_batch_get_variant(const bnz_batch* b, int* v) {
  if (!b || !v) return BNZ_ERR_ARG;
  *v = b->variant;
  return BNZ_OK;
}

// Time `steps` batch steps of variant v (after one untimed step) on the live
// state, then put the state, the time records and the variant back.
int bnz_batch_time_variant(bnz_batch* b, int v, int steps, double* ms) {
  if (!b || steps < 1) return BNZ_ERR_ARG;
  if (b->dims3) return bfail(b, BNZ_ERR_UNSUPPORTED, "3D batches have one kernel shape");
  const int v0 = b->variant, p0 = b->parity;
  int rc = bnz_batch_set_variant(b, v);
  if (rc) return rc;
  // save every instance's state of the current parity and its time record
  std::vector<double*> saved(b->ctx.size(), nullptr);
  std::vector<DtState> dts(b->ctx.size());
  for (size_t q = 0; q < b->ctx.size(); ++q) {
    bnz_ctx* c = b->ctx[q];
    size_t n9 = 9 * c->ncell, n3 = 3 * c->ncell;
    CKB(cudaMalloc((void**)&saved[q], (n9 + n3) * sizeof(double)));
    CKB(cudaMemcpyAsync(saved[q], c->wbuf[p0], n9 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    CKB(cudaMemcpyAsync(saved[q] + n9, c->bbuf[p0], n3 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    CKB(cudaMemcpyAsync(&dts[q], c->d_ds, sizeof(DtState), cudaMemcpyDeviceToHost, b->stream));
  }
  CKB(cudaStreamSynchronize(b->stream));
  // the trial must really step: no tmax clip (the time records are restored below)
  {
    const int n = (int)b->ctx.size();
    k_set_tmax<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_inst, n, 1e300);
    CKB(cudaGetLastError());
  }
  const int mode = b->md.fixdt ? FDT_FIXED : FDT_CFL;
  cudaEvent_t e0, e1;
  CKB(cudaEventCreate(&e0));
  CKB(cudaEventCreate(&e1));
  int p = p0;
  for (int s = 0; s <= steps; ++s) {
    if (s == 1) CKB(cudaEventRecord(e0, b->stream));
    b->L->fused_step(batch_launch(b, mode), p);
    p ^= 1;
  }
  CKB(cudaEventRecord(e1, b->stream));
  CKB(cudaEventSynchronize(e1));
  float t = 0.f;
  CKB(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t / steps;
  for (size_t q = 0; q < b->ctx.size(); ++q) {
    bnz_ctx* c = b->ctx[q];
    size_t n9 = 9 * c->ncell, n3 = 3 * c->ncell;
    CKB(cudaMemcpyAsync(c->wbuf[p0], saved[q], n9 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    CKB(cudaMemcpyAsync(c->bbuf[p0], saved[q] + n9, n3 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    CKB(cudaMemcpyAsync(c->d_ds, &dts[q], sizeof(DtState), cudaMemcpyHostToDevice, b->stream));
  }
  CKB(cudaStreamSynchronize(b->stream));
  for (double* ptr : saved) cudaFree(ptr);
  b->parity = p0;
  for (bnz_ctx* c : b->ctx) set_parity(c, p0);
  return bnz_batch_set_variant(b, v0);
}

int bnz_batch_autotune(bnz_batch* b, int steps, int* best, double* ms_per_variant) {
  if (!b) return BNZ_ERR_ARG;
  if (b->dims3) return bfail(b, BNZ_ERR_UNSUPPORTED, "3D batches have one kernel shape");
  const bool hlld = b->md.rsolver == BNZ_RS_HLLD;
  double best_ms = 1e300;
  int bv = 0;
  for (int v = 0; v < FUSED_NVARIANT; ++v) {
    double ms = -1.;
    if (fused_variant_built(v, hlld)) {
      int rc = bnz_batch_time_variant(b, v, steps, &ms);
      if (rc) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        bv = v;
      }
    }
    if (ms_per_variant) ms_per_variant[v] = ms;
  }
  if (best) *best = bv;
  return bnz_batch_set_variant(b, bv);
}

}  // extern "C"
