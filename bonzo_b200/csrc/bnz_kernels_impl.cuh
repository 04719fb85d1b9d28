// bnz_kernels_impl.cuh -- kernels and their host launchers, compiled once per
// floating-point mode: bnz_kernels_exact.cu (no multiply-add contraction, the
// bit-for-bit parity build) and bnz_kernels_fast.cu (DFMA contraction).
// The including file defines BNZ_NS (the namespace name).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "bnz_common.h"
#include "bnz_launch.h"

namespace BNZ_NS {

#include "bnz_device.cuh"
#include "bnz_plain.cuh"
#include "bnz_bc_dt.cuh"
#include "bnz_diffusion.cuh"
#include "bnz_source.cuh"
#include "bnz_split.cuh"
#include "bnz_fused.cuh"
#include "bnz_fused3d.cuh"
#include "bnz_split_tma.cuh"
#include "bnz_adjoint_math.h"
#include "bnz_adjoint.cuh"

namespace {

inline int nblocks(long long n, int threads, int cap = 148 * 32) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

inline plain::Box mkbox(int x0, int x1, int y0, int y1, int z0, int z1) {
  plain::Box b;
  b.lo = make_int3(x0, y0, z0);
  b.hi = make_int3(x1, y1, z1);
  return b;
}

inline long long boxn(const plain::Box& b) {
  return (long long)(b.hi.x - b.lo.x + 1) * (b.hi.y - b.lo.y + 1) * (b.hi.z - b.lo.z + 1);
}

// integrator.pyx:375-383
inline void integr_lims(const GridDev& g, int order, int* l) {
  const int N[3] = {g.nx, g.ny, g.nz};
  for (int a = 0; a < 3; ++a) {
    l[2 * a] = order + 1;
    l[2 * a + 1] = N[a] - 2 - order;
  }
  if (g.dims < 2) l[2] = l[3] = 0;
  if (g.dims < 3) l[4] = l[5] = 0;
}

template <int AX, int ORDER>
int launch_flux_rs(const StepArgs& a, const double* w, const double* bf, const plain::Box& b) {
  const int T = 128;
  int nb = nblocks(boxn(b), T);
  switch (a.rsolver) {
    case dev::RS_HLLD:
      plain::k_flux<AX, ORDER, dev::RS_HLLD><<<nb, T, 0, a.stream>>>(a.g, w, bf, a.flx[AX], b, a.limiter, a.charact_proj,
                                                                  a.err);
      break;
    case dev::RS_HLLT:
      plain::k_flux<AX, ORDER, dev::RS_HLLT><<<nb, T, 0, a.stream>>>(a.g, w, bf, a.flx[AX], b, a.limiter, a.charact_proj,
                                                                  a.err);
      break;
    case dev::RS_HLLC:
      plain::k_flux<AX, ORDER, dev::RS_HLLC><<<nb, T, 0, a.stream>>>(a.g, w, bf, a.flx[AX], b, a.limiter, a.charact_proj,
                                                                  a.err);
      break;
    case dev::RS_HLL_HYDRO:
      plain::k_flux<AX, ORDER, dev::RS_HLL_HYDRO><<<nb, T, 0, a.stream>>>(a.g, w, bf, a.flx[AX], b, a.limiter,
                                                                       a.charact_proj, a.err);
      break;
    default:
      plain::k_flux<AX, ORDER, dev::RS_HLL><<<nb, T, 0, a.stream>>>(a.g, w, bf, a.flx[AX], b, a.limiter, a.charact_proj,
                                                                  a.err);
      break;
  }
  return 1;
}

template <int AX>
int launch_flux(const StepArgs& a, int order, const double* w, const double* bf, const plain::Box& b) {
  if (order == 0) return launch_flux_rs<AX, 0>(a, w, bf, b);
  return launch_flux_rs<AX, 1>(a, w, bf, b);
}

// godunov.pyx:20-209 + 215-252 (integrate_hydro, integrator.pyx:51-79)
int integrate_hydro(const StepArgs& a, double* u1, const double* u0, const double* w0, const double* b0, int order,
                     const double* dtp, double fac) {
  const GridDev& g = a.g;
  int l[6];
  integr_lims(g, order, l);
  int il = l[0], iu = l[1], jl = l[2], ju = l[3], kl = l[4], ku = l[5];
  int nl = 0;
  {  // x faces il..iu+1 on rows jl-1..ju+1, kl-1..ku+1
    int jb = jl - 1, je = ju + 1, kb = kl - 1, ke = ku + 1;
    if (g.dims < 2) jb = je = 0;
    if (g.dims < 3) kb = ke = 0;
    nl += launch_flux<0>(a, order, w0, b0, mkbox(il, iu + 1, jb, je, kb, ke));
  }
  if (g.dims >= 2) {
    int kb = kl - 1, ke = ku + 1;
    if (g.dims < 3) kb = ke = 0;
    nl += launch_flux<1>(a, order, w0, b0, mkbox(il - 1, iu + 1, jl, ju + 1, kb, ke));
  }
  if (g.dims >= 3) nl += launch_flux<2>(a, order, w0, b0, mkbox(il - 1, iu + 1, jl - 1, ju + 1, kl, ku + 1));
  plain::Box b = mkbox(il, iu, jl, ju, kl, ku);
  plain::k_advance_hydro<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, u1, u0, a.flx[0], a.flx[1], a.flx[2], b,
                                                                        dtp, fac);
  return nl + 1;
}

// integrator.pyx:85-126
int integrate_field(const StepArgs& a, double* u1, double* b1, const double* w0, const double* b0, int order,
                     const double* dtp, double fac) {
  const GridDev& g = a.g;
  int l[6];
  integr_lims(g, order, l);
  {
    int il = l[0] - 1, iu = l[1] + 1, jl = l[2] - 1, ju = l[3] + 1, kl = l[4] - 1, ku = l[5] + 1;
    if (g.dims < 2) jl = ju = 0;
    if (g.dims < 3) kl = ku = 0;
    plain::Box b = mkbox(il, iu, jl, ju, kl, ku);
    plain::k_ec<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, w0, a.ec, b);
  }
  {
    int il = l[0], iu = l[1] + 1, jl = l[2], ju = l[3] + 1, kl = l[4], ku = l[5] + 1;
    if (g.dims < 2) jl = ju = 0;
    if (g.dims < 3) kl = ku = 0;
    plain::Box b = mkbox(il, iu, jl, ju, kl, ku);
    plain::k_ee<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, a.ec, a.flx[0], a.flx[1], a.flx[2], a.ee, b);
  }
  {
    plain::Box bx = mkbox(l[0], l[1] + 1, l[2], l[3], l[4], l[5]);
    // y faces to lims[3]+1 like x and z (the reference's ct.pyx:48 stops at
    // lims[3] and leaves the top predictor face stale)
    plain::Box by = mkbox(l[0], l[1], l[2], g.dims >= 2 ? l[3] + 1 : l[3], l[4], l[5]);
    plain::Box bz = mkbox(l[0], l[1], l[2], l[3], l[4], g.dims >= 3 ? l[5] + 1 : l[5]);
    plain::k_advance_b<0><<<nblocks(boxn(bx), 256), 256, 0, a.stream>>>(g, b1, b0, a.ee, bx, dtp, fac);
    plain::k_advance_b<1><<<nblocks(boxn(by), 256), 256, 0, a.stream>>>(g, b1, b0, a.ee, by, dtp, fac);
    plain::k_advance_b<2><<<nblocks(boxn(bz), 256), 256, 0, a.stream>>>(g, b1, b0, a.ee, bz, dtp, fac);
  }
  plain::Box b = mkbox(l[0], l[1], l[2], l[3], l[4], l[5]);
  plain::k_interp_bc<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, u1, b1, b);
  return 6;
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers exported to the host context (declared in bnz_launch.h).
// ---------------------------------------------------------------------------

// integrator.pyx:132-170 add_source_terms on the stage's update range
int source(const StepArgs& a, double* u1, const double* w0, int order, const double* dtp, double fac) {
  int l[6];
  integr_lims(a.g, order, l);
  plain::Box b = mkbox(l[0], l[1], l[2], l[3], l[4], l[5]);
  srcterm::k_source<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(a.g, u1, w0, a.fdriv, a.grav[0], a.grav[1],
                                                                  a.grav[2], b, dtp, fac);
  return 1;
}

// integrator.pyx:176-194 update_physics: the driving force on the predictor range
int drive(const StepArgs& a, const DriveArgs& d, const double* dtp) {
  int l[6];
  integr_lims(a.g, 0, l);
  plain::Box b = mkbox(l[0], l[1], l[2], l[3], l[4], l[5]);
  srcterm::k_drive<<<nblocks(boxn(b), 128), 128, 0, a.stream>>>(a.g, d.fdriv, d.modes, d.nmod, d.k0[0], d.k0[1],
                                                                 d.k0[2], d.tau, d.f0, b, dtp);
  return 1;
}

namespace {
// The reference's C-level Riemann call (fluxes_c.h:3-20: flux rows from wL / wR
// rows and the face-normal field bx over i1..i2) on device rows: entry q of
// row n at [n * count + q].  nvar = 9 (MHD: wL[BX] = wR[BX] = bx) or 6 (the
// hydro build: the field entries are zero and not stored).
template <int RS>
__global__ void k_riemann_rows(const double* __restrict__ wl, const double* __restrict__ wr,
                               const double* __restrict__ bx, double* __restrict__ flux, int count, int nvar,
                               double gam, unsigned* err) {
  unsigned e = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    double wL[dev::NM], wR[dev::NM], f[dev::NM];
#pragma unroll
    for (int n = 0; n < dev::NM; ++n) {
      wL[n] = n < nvar ? wl[(long long)n * count + q] : 0.;
      wR[n] = n < nvar ? wr[(long long)n * count + q] : 0.;
    }
    if (nvar == dev::NM) wL[dev::BX] = wR[dev::BX] = bx[q];
    dev::riemann<RS>(f, wL, wR, gam, e);
#pragma unroll
    for (int n = 0; n < dev::NM; ++n)
      if (n < nvar) flux[(long long)n * count + q] = f[n];
  }
  if (e && err) atomicOr(err, e);
}
}  // namespace

int riemann_rows(int rs, const double* wl, const double* wr, const double* bx, double* flux, int n, int nvar,
                 double gam, unsigned* err, cudaStream_t s) {
  const int T = 128, nb = nblocks(n, T);
  switch (rs) {
    case dev::RS_HLLD: k_riemann_rows<dev::RS_HLLD><<<nb, T, 0, s>>>(wl, wr, bx, flux, n, nvar, gam, err); break;
    case dev::RS_HLLT: k_riemann_rows<dev::RS_HLLT><<<nb, T, 0, s>>>(wl, wr, bx, flux, n, nvar, gam, err); break;
    case dev::RS_HLLC: k_riemann_rows<dev::RS_HLLC><<<nb, T, 0, s>>>(wl, wr, bx, flux, n, nvar, gam, err); break;
    case dev::RS_HLL_HYDRO:
      k_riemann_rows<dev::RS_HLL_HYDRO><<<nb, T, 0, s>>>(wl, wr, bx, flux, n, nvar, gam, err);
      break;
    default: k_riemann_rows<dev::RS_HLL><<<nb, T, 0, s>>>(wl, wr, bx, flux, n, nvar, gam, err); break;
  }
  return 1;
}

int plain_predictor_corrector(const StepArgs& a, const double* dtp) {
  const GridDev& g = a.g;
  int l[6];
  // predictor (vanleer.pyx:104-120): order 0, dt/2, Us from U, W, B
  int nl = integrate_hydro(a, a.cons_s, a.cons, a.prim, a.bfld, 0, dtp, 0.5);
  // the hydro build has no field to transport (vanleer.pyx:110-112 under MFIELD)
  if (!a.hydro) nl += integrate_field(a, a.cons_s, a.bfld_s, a.prim, a.bfld, 0, dtp, 0.5);
  if (a.src) nl += source(a, a.cons_s, a.prim, 0, dtp, 0.5);
  integr_lims(g, 0, l);
  {
    plain::Box b = mkbox(l[0], l[1], l[2], l[3], l[4], l[5]);
    plain::k_cons2prim<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, a.prim, a.cons_s, b, a.err);
  }
  // corrector (vanleer.pyx:130-151): order reconstr_order, dt, U from Ws, Bs
  int order = a.reconstr_order;
  nl += integrate_hydro(a, a.cons, a.cons, a.prim, a.bfld_s, order, dtp, 1.0);
  if (!a.hydro) nl += integrate_field(a, a.cons, a.bfld, a.prim, a.bfld, order, dtp, 1.0);
  if (a.src) nl += source(a, a.cons, a.prim, order, dtp, 1.0);
  integr_lims(g, order, l);
  {
    plain::Box b = mkbox(l[0], l[1], l[2], l[3], l[4], l[5]);
    plain::k_cons2prim<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, a.prim, a.cons, b, a.err);
  }
  return nl + 2;
}

// SM count of the current device (cached per device).
inline int sm_count() {
  static int nsm[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!nsm[dev]) cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, nsm[dev]);
}

namespace {
// Blocks of 32 x 8 cells of the box, split::UPD_KZ z indices each.
inline dim3 cell_grid(const plain::Box& b) {
  const int kz = split::UPD_KZ;
  return dim3((b.hi.x - b.lo.x + 32) / 32, (b.hi.y - b.lo.y + 8) / 8, (b.hi.z - b.lo.z + kz) / kz);
}

// The prim arrays a split stage reads: w on [vlo, vhi], wfb elsewhere.
struct SplitSrc {
  const double* w;
  const double* wfb;
  int3 vlo, vhi;
};

// The corrector's PLM fluxes of a 3D grid with tensor maps: a persistent
// kernel of two blocks per SM (at most one per tile), each tile one TMA box of
// the predictor's prim (x sweep: first face column even).
template <int AX, int RS>
void launch_flux_tma(const StepArgs& a, const SplitSrc& s, const double* bf, const plain::Box& b, unsigned nblk) {
  constexpr size_t sm = sizeof(split::FluxSmem<AX>);
  static bool attr = false;  // once per kernel
  if (!attr) {
    cudaFuncSetAttribute(split::k_flux_tile_tma<AX, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  split::k_flux_tile_tma<AX, RS><<<nblk, 256, sm, a.stream>>>(a.g, a.smaps, s.wfb, s.vlo, s.vhi, bf, a.flx[AX], b,
                                                              a.limiter, a.charact_proj, a.err);
}

template <int AX>
int split_flux_tma(const StepArgs& a, const SplitSrc& s, const double* bf, const plain::Box& b) {
  using T = split::FTT<AX>;
  const int lo[3] = {b.lo.x, b.lo.y, b.lo.z}, hi[3] = {b.hi.x, b.hi.y, b.hi.z};
  const int lb0 = AX == 0 ? lo[T::TAX] : (lo[T::TAX] & ~1);
  const long long na = (hi[AX] - lo[AX] + T::NA) / T::NA, nb = (hi[T::TAX] - lb0 + T::NB) / T::NB;
  const long long ntile = na * nb * (hi[T::OAX] - lo[T::OAX] + 1);
  const unsigned nblk = (unsigned)std::min<long long>(ntile, 2LL * sm_count());
  switch (a.rsolver) {
    case dev::RS_HLLD: launch_flux_tma<AX, dev::RS_HLLD>(a, s, bf, b, nblk); break;
    case dev::RS_HLLT: launch_flux_tma<AX, dev::RS_HLLT>(a, s, bf, b, nblk); break;
    case dev::RS_HLLC: launch_flux_tma<AX, dev::RS_HLLC>(a, s, bf, b, nblk); break;
    case dev::RS_HLL_HYDRO: launch_flux_tma<AX, dev::RS_HLL_HYDRO>(a, s, bf, b, nblk); break;
    default: launch_flux_tma<AX, dev::RS_HLL>(a, s, bf, b, nblk); break;
  }
  return 1;
}

template <int AX, int ORDER>
int split_flux(const StepArgs& a, const SplitSrc& s, const double* bf, const plain::Box& b) {
  using T = split::FT<AX>;
  if (ORDER == 1 && a.g.dims == 3 && a.smaps && s.w == a.cons_s && (AX != 0 || (b.lo.x & 1) == 0))
    return split_flux_tma<AX>(a, s, bf, b);
  const int lo[3] = {b.lo.x, b.lo.y, b.lo.z}, hi[3] = {b.hi.x, b.hi.y, b.hi.z};
  const long long na = (hi[AX] - lo[AX] + T::NA) / T::NA, nb = (hi[T::TAX] - lo[T::TAX] + T::NB) / T::NB;
  const unsigned nblk = (unsigned)(na * nb * (hi[T::OAX] - lo[T::OAX] + 1));
  switch (a.rsolver) {
    case dev::RS_HLLD:
      split::k_flux_tile<AX, ORDER, dev::RS_HLLD><<<nblk, T::NT, 0, a.stream>>>(
          a.g, s.w, s.wfb, s.vlo, s.vhi, bf, a.flx[AX], b, a.limiter, a.charact_proj, a.err);
      break;
    case dev::RS_HLLT:
      split::k_flux_tile<AX, ORDER, dev::RS_HLLT><<<nblk, T::NT, 0, a.stream>>>(
          a.g, s.w, s.wfb, s.vlo, s.vhi, bf, a.flx[AX], b, a.limiter, a.charact_proj, a.err);
      break;
    case dev::RS_HLLC:
      split::k_flux_tile<AX, ORDER, dev::RS_HLLC><<<nblk, T::NT, 0, a.stream>>>(
          a.g, s.w, s.wfb, s.vlo, s.vhi, bf, a.flx[AX], b, a.limiter, a.charact_proj, a.err);
      break;
    case dev::RS_HLL_HYDRO:
      split::k_flux_tile<AX, ORDER, dev::RS_HLL_HYDRO><<<nblk, T::NT, 0, a.stream>>>(
          a.g, s.w, s.wfb, s.vlo, s.vhi, bf, a.flx[AX], b, a.limiter, a.charact_proj, a.err);
      break;
    default:
      split::k_flux_tile<AX, ORDER, dev::RS_HLL><<<nblk, T::NT, 0, a.stream>>>(
          a.g, s.w, s.wfb, s.vlo, s.vhi, bf, a.flx[AX], b, a.limiter, a.charact_proj, a.err);
      break;
  }
  return 1;
}

// Donor-cell fluxes from one prim array go through plain::k_flux: with no
// slopes to share, staging the cells in shared memory only adds a barrier
// (the split tile kernel measured about 9 % slower there).
template <int AX>
int split_flux(const StepArgs& a, int order, const SplitSrc& s, const double* bf, const plain::Box& b) {
  if (order == 0 && s.w == s.wfb) return launch_flux<AX>(a, 0, s.w, bf, b);
  return order == 0 ? split_flux<AX, 0>(a, s, bf, b) : split_flux<AX, 1>(a, s, bf, b);
}

// One VL2 stage on the split path (vanleer.pyx:104-120 or 130-151): the face
// fluxes over the boxes of integrate_hydro, the edge EMFs over the box of
// integrate_field, then the fused update of the stage's range from U^n =
// prim2cons(a.prim) into w1.
int split_stage(const StepArgs& a, const SplitSrc& s, double* w1, double* b1, const double* b0, double* bsave,
                const double* bf, int order, const double* dtp, double fac) {
  const GridDev& g = a.g;
  int l[6];
  integr_lims(g, order, l);
  const int il = l[0], iu = l[1], jl = l[2], ju = l[3], kl = l[4], ku = l[5];
  const int jb = g.dims >= 2 ? jl - 1 : 0, je = g.dims >= 2 ? ju + 1 : 0;
  const int kb = g.dims >= 3 ? kl - 1 : 0, ke = g.dims >= 3 ? ku + 1 : 0;
  int nl = split_flux<0>(a, order, s, bf, mkbox(il, iu + 1, jb, je, kb, ke));
  if (g.dims >= 2) nl += split_flux<1>(a, order, s, bf, mkbox(il - 1, iu + 1, jl, ju + 1, kb, ke));
  if (g.dims >= 3) nl += split_flux<2>(a, order, s, bf, mkbox(il - 1, iu + 1, jl - 1, ju + 1, kl, ku + 1));
  {
    plain::Box b = mkbox(il, iu + 1, jl, g.dims >= 2 ? ju + 1 : 0, kl, g.dims >= 3 ? ku + 1 : 0);
    split::k_ee<<<cell_grid(b), dim3(32, 8), 0, a.stream>>>(g, s.w, s.wfb, s.vlo, s.vhi, a.flx[0], a.flx[1],
                                                             a.flx[2], a.ee, b);
  }
  plain::Box b = mkbox(il, iu, jl, ju, kl, ku);
  if (g.dims == 3 && a.smaps) {
    // the TMA-fed form (3D, even Ntot_x): blocks of 32 x 8 columns from an
    // even first column, split::UPD_KZ planes each
    constexpr size_t sm = sizeof(split::TmaSmem);
    static bool attr = false;  // once per floating-point build
    if (!attr) {
      cudaFuncSetAttribute(split::k_update_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      attr = true;
    }
    const int x0base = b.lo.x & ~1;
    const dim3 grid((b.hi.x - x0base + 32) / 32, (b.hi.y - b.lo.y + 8) / 8,
                    (b.hi.z - b.lo.z + split::UPD_KZ) / split::UPD_KZ);
    const int b0map = b0 == a.bfld ? split::TM_BFLD : split::TM_BSAVE;
    split::k_update_tma<<<grid, dim3(32, 8), sm, a.stream>>>(g, w1, s.w, b1, bsave, a.smaps, b0map, b, x0base, dtp,
                                                             fac, a.src, a.grav[0], a.grav[1], a.grav[2], a.fdriv,
                                                             a.err);
    return nl + 2;
  }
  split::k_update<<<cell_grid(b), dim3(32, 8), 0, a.stream>>>(
      g, w1, a.prim, s.w, b1, b0, bsave, a.flx[0], a.flx[1], a.flx[2], a.ee, b, dtp, fac, a.src, a.grav[0],
      a.grav[1], a.grav[2], a.fdriv, a.err);
  return nl + 2;
}
}  // namespace

// vanleer.pyx:101-151 on the split path.  The predictor writes W^(n+1/2) to
// a.cons_s (cells 1..Ntot-2 of each active axis), so that a.prim keeps W^n for
// the corrector's U^n; the corrector reads W^(n+1/2) there and W^n on the
// outer cells, as the plain path's in-place prim holds them.  The predictor
// also saves the faces of b^n it reads into the spare face array a.ec (the
// split path forms the cell EMFs on the fly), so that the corrector can
// update a.bfld in place of a neighbour's reads: it reads b^n from the copy.
// The conserved state is not written: the context forms it from prim after
// the boundary fill, when it is asked for.  In the hydro build (field entries
// and face field held at zero, the hydro solvers' field fluxes zero) the same
// launches run and the field stays zero.
int split_predictor_corrector(const StepArgs& a, const double* dtp) {
  const GridDev& g = a.g;
  const int N[3] = {g.nx, g.ny, g.nz};
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = d < g.dims ? 1 : 0;
    hi[d] = d < g.dims ? N[d] - 2 : 0;
  }
  const SplitSrc pred = {a.prim, a.prim, make_int3(0, 0, 0), make_int3(g.nx - 1, g.ny - 1, g.nz - 1)};
  const SplitSrc corr = {a.cons_s, a.prim, make_int3(lo[0], lo[1], lo[2]), make_int3(hi[0], hi[1], hi[2])};
  int nl = split_stage(a, pred, a.cons_s, a.bfld_s, a.bfld, a.ec, a.bfld, 0, dtp, 0.5);
  nl += split_stage(a, corr, a.prim, a.bfld, a.ec, nullptr, a.bfld_s, a.reconstr_order, dtp, 1.0);
  return nl;
}

int apply_bc(const StepArgs& a, double* prim, double* bfld, unsigned mask) {
  const GridDev& g = a.g;
  bcdt::FieldList fl;
  fl.n = 0;
  for (int f = 0; f < 12; ++f)
    if (mask & (1u << f)) fl.f[fl.n++] = f;
  if (fl.n == 0) return 0;
  int nl = 0;
  for (int ax = 2; ax >= 0; --ax) {
    if (ax >= g.dims) continue;
    const int N[3] = {g.nx, g.ny, g.nz};
    long long nother = (long long)N[ax == 0 ? 1 : 0] * N[ax == 2 ? 1 : 2];
    long long n = 2LL * g.ng * nother;
    dim3 grid(nblocks(n, 256, 4096), fl.n);
    bcdt::k_bc_axis<<<grid, 256, 0, a.stream>>>(g, ax, prim, bfld, fl, a.bc[ax][0], a.bc[ax][1], a.face_aware);
    ++nl;
  }
  return nl;
}

int prim2cons_all(const StepArgs& a) {
  const GridDev& g = a.g;
  plain::Box b = mkbox(0, g.nx - 1, 0, g.ny - 1, 0, g.nz - 1);
  plain::k_prim2cons<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, a.cons, a.prim, b);
  return 1;
}

int cons2prim_all(const StepArgs& a) {
  const GridDev& g = a.g;
  plain::Box b = mkbox(0, g.nx - 1, 0, g.ny - 1, 0, g.nz - 1);
  plain::k_cons2prim<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, a.prim, a.cons, b, a.err);
  return 1;
}

int interp_bc_active(const StepArgs& a) {
  const GridDev& g = a.g;
  plain::Box b = mkbox(g.i1, g.i2, g.j1, g.j2, g.k1, g.k2);
  plain::k_interp_bc<<<nblocks(boxn(b), 256), 256, 0, a.stream>>>(g, a.prim, a.bfld, b);
  return 1;
}

int new_dt(const StepArgs& a, const double* prim, DtState* ds, double cour, int clip) {
  const GridDev& g = a.g;
  long long n = (long long)(g.i2 - g.i1 + 1) * (g.j2 - g.j1 + 1) * (g.k2 - g.k1 + 1);
  bcdt::k_dt_reset<<<1, 1, 0, a.stream>>>(ds);
  bcdt::k_cds_max<<<nblocks(n, 256, 148 * 8), 256, 0, a.stream>>>(g, prim, &ds->cdsmax_bits, a.hydro);
  bcdt::k_dt_finalize<<<1, 1, 0, a.stream>>>(ds, cour, clip);
  return 3;
}

int set_dt(cudaStream_t s, DtState* ds, double dt) {
  bcdt::k_dt_set<<<1, 1, 0, s>>>(ds, dt);
  return 1;
}

int fixed_dt(cudaStream_t s, DtState* ds, double dt) {
  bcdt::k_dt_fixed<<<1, 1, 0, s>>>(ds, dt);
  return 1;
}
int time_advance(cudaStream_t s, DtState* ds) {
  bcdt::k_time_advance<<<1, 1, 0, s>>>(ds);
  return 1;
}

// --- conduction ---------------------------------------------------------

int diff_dt_max(const StepArgs& a, const DiffArgs& d, unsigned long long* slot) {
  const GridDev& g = a.g;
  long long n = (long long)(g.i2 - g.i1 + 1) * (g.j2 - g.j1 + 1) * (g.k2 - g.k1 + 1);
  diff::k_diff_dt_max<<<nblocks(n, 256, 148 * 8), 256, 0, a.stream>>>(g, a.prim, d.kappa0, slot);
  return 1;
}

// One RKL2 stage (thcond_elec.pyx:75-94 with the operator of :118-338):
// T = p / rho on every cell, then the fused flux / divergence / update pass on
// cells 1..Ntot-2 of every active axis.
int diff_stage(const StepArgs& a, const DiffArgs& d, int first, const double* coef, const double* dtp) {
  const GridDev& g = a.g;
  diff::k_temp<<<nblocks(g.sv, 256), 256, 0, a.stream>>>(g, a.prim, d.temp);
  int il = 1, iu = g.nx - 2;
  int jl = g.dims >= 2 ? 1 : 0, ju = g.dims >= 2 ? g.ny - 2 : 0;
  int kl = g.dims >= 3 ? 1 : 0, ku = g.dims >= 3 ? g.nz - 2 : 0;
  int3 lo = make_int3(il, jl, kl), hi = make_int3(iu, ju, ku);
  long long n = (long long)(hi.x - lo.x + 1) * (hi.y - lo.y + 1) * (hi.z - lo.z + 1);
  if (g.dims == 3) {
    // tiles of 8 x 8 x 8 cells: every face flux formed once per tile
    const int nb = ((hi.x - lo.x + 8) / 8) * ((hi.y - lo.y + 8) / 8) * ((hi.z - lo.z + 8) / 8);
    diff::k_stage_tile<8, 8, 8><<<nb, 512, 0, a.stream>>>(g, a.prim, a.bfld, d.temp, d, lo, hi, first, coef[0],
                                                          coef[1], coef[2], coef[3], dtp);
  } else {
    diff::k_stage<<<nblocks(n, 256), 256, 0, a.stream>>>(g, a.prim, a.bfld, d.temp, d, lo, hi, first, coef[0],
                                                          coef[1], coef[2], coef[3], dtp);
  }
  return 2;
}

// --- fused 2D path (one launch per stage for the whole batch) --------------

namespace {

template <int TX, int TY, int RS, int LIM>
void launch_corr(const FusedLaunch& f, int parity) {
  constexpr size_t smB = fused::Smem<TX, TY, 2>::bytes;
  static bool attrs = false;
  if (!attrs) {
    cudaFuncSetAttribute(fused::k_corr2d<TX, TY, RS, LIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smB);
    attrs = true;
  }
  fused::k_corr2d<TX, TY, RS, LIM><<<f.ntB, 256, smB, f.stream>>>(f.insts, f.tilesB, parity, f.charact_proj);
}

// Persistent corrector: (SMs x resident blocks) blocks, never more than tiles.
template <int TX, int TY, int RS, int LIM>
void launch_corr_pq(const FusedLaunch& f, int parity) {
  constexpr size_t sm = fused::TmaBox<TX, TY>::smem_bytes;
  static int per_sm = 0;
  if (!per_sm) {
    cudaFuncSetAttribute(fused::k_corr2d_pq<TX, TY, RS, LIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused::k_corr2d_pq<TX, TY, RS, LIM>, 256, sm);
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = std::min(f.ntB, per_sm * sm_count());
  if (grid < 1) return;
  fused::k_corr2d_pq<TX, TY, RS, LIM><<<grid, 256, sm, f.stream>>>(f.insts, f.tilesB, f.ntB, parity,
                                                                    f.charact_proj, f.wsmaps, f.queue, f.withhold);
}

template <int TX, int TY, int RS>
void launch_pred_pq(const FusedLaunch& f, int parity) {
  constexpr size_t sm = fused::TmaBoxP<TX, TY>::smem_bytes;
  static int per_sm = 0;
  if (!per_sm) {
    cudaFuncSetAttribute(fused::k_pred2d_pq<TX, TY, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused::k_pred2d_pq<TX, TY, RS>, 256, sm);
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = std::min(f.ntA, per_sm * sm_count());
  if (grid < 1) return;
  fused::k_pred2d_pq<TX, TY, RS><<<grid, 256, sm, f.stream>>>(f.insts, f.tilesA, f.ntA, parity, f.wmaps,
                                                              f.queue + 1, f.withhold);
}

template <int TX, int TY, int RS, int LIM>
void launch_corr_any(const FusedLaunch& f, int parity) {
  if constexpr ((TX == 15 && TY == 14) || (TX == 14 && TY == 14)) {
    if (f.wsmaps && f.queue) {
      launch_corr_pq<TX, TY, RS, LIM>(f, parity);
      return;
    }
  }
  launch_corr<TX, TY, RS, LIM>(f, parity);
}

template <int TX, int TY, int RS, int STAGED>
void launch_variant(const FusedLaunch& f, int parity) {
  constexpr int TXA = TX + 4, TYA = TY + 4;  // predictor tiles grow by the ghost rings
  constexpr size_t smA = fused::Smem<TXA, TYA, STAGED ? 1 : 0>::bytes;
  static bool attrs = false;
  if (!attrs) {
    cudaFuncSetAttribute(fused::k_pred2d<TXA, TYA, RS, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smA);
    attrs = true;
  }
  if (f.events) cudaEventRecord(f.events[1], f.stream);
  bool done = false;
  if constexpr (((TX == 15 && TY == 14) || (TX == 14 && TY == 14)) && STAGED == 0) {
    if (f.wmaps && f.queue) {
      launch_pred_pq<TX, TY, RS>(f, parity);
      done = true;
    }
  }
  if (!done)
    fused::k_pred2d<TXA, TYA, RS, STAGED><<<f.ntA, 256, smA, f.stream>>>(f.insts, f.tilesA, parity, f.limiter);
  if (f.events) cudaEventRecord(f.events[2], f.stream);
  // the limiter is a compile-time choice of the corrector (reconstr_c.h:28-44)
  if (f.limiter == dev::LIM_MC) launch_corr_any<TX, TY, RS, dev::LIM_MC>(f, parity);
  else if (f.limiter == dev::LIM_MM) launch_corr_any<TX, TY, RS, dev::LIM_MM>(f, parity);
  else launch_corr_any<TX, TY, RS, dev::LIM_VL>(f, parity);
  if (f.events) cudaEventRecord(f.events[3], f.stream);
}

template <int RS>
void launch_pred_corr(const FusedLaunch& f, int parity) {
  // FUSED_VARIANTS in bnz_common.h; variants 1-7 are built for HLLD only
  if constexpr (RS != dev::RS_HLLD) {
    if (f.variant == 8) {
      launch_variant<15, 14, RS, 0>(f, parity);  // persistent predictor and corrector
      return;
    }
    if (f.variant == 9) {
      launch_variant<14, 14, RS, 0>(f, parity);
      return;
    }
  }
  if constexpr (RS == dev::RS_HLLD) {
    switch (f.variant) {
      case 1: launch_variant<32, 8, RS, 1>(f, parity); return;
      case 2: launch_variant<16, 16, RS, 0>(f, parity); return;
      case 3: launch_variant<16, 16, RS, 1>(f, parity); return;
      case 4: launch_variant<15, 14, RS, 0>(f, parity); return;
      case 5: launch_variant<15, 14, RS, 1>(f, parity); return;
      case 6: launch_variant<15, 14, RS, 0>(f, parity); return;  // persistent corrector when maps are given
      case 7: launch_variant<15, 14, RS, 1>(f, parity); return;
      case 8: launch_variant<15, 14, RS, 0>(f, parity); return;  // persistent predictor too
      case 9: launch_variant<14, 14, RS, 0>(f, parity); return;
      default: break;
    }
  }
  launch_variant<32, 8, RS, 0>(f, parity);
}
}  // namespace

int fused_step(const FusedLaunch& f, int parity) {
  if (f.events) cudaEventRecord(f.events[0], f.stream);
  fused::k_dt_batch<<<(f.ninst + 127) / 128, 128, 0, f.stream>>>(f.insts + f.inst0, f.ninst, parity, f.cour,
                                                                  f.dt_mode, f.dt_fixed, f.queue);
  switch (f.rsolver) {
    case dev::RS_HLLD: launch_pred_corr<dev::RS_HLLD>(f, parity); break;
    case dev::RS_HLLT: launch_pred_corr<dev::RS_HLLT>(f, parity); break;
    default: launch_pred_corr<dev::RS_HLL>(f, parity); break;
  }
  return 3;
}

int fused_time(const FusedLaunch& f) {
  fused::k_time_batch<<<(f.ninst + 127) / 128, 128, 0, f.stream>>>(f.insts + f.inst0, f.ninst);
  return 1;
}

// CFL max of the current state into slot `parity` (needed before the first
// fused step and after the state was replaced or diffused).
int fused_cds(const FusedLaunch& f, int parity) {
  fused::k_cds_batch<<<f.ntB, 256, 0, f.stream>>>(f.insts, f.tilesB, parity);
  return 1;
}

// --- fused 3D path (z-marching chunks, one launch per stage) -----------------

namespace {

template <int ORDER, int RS, int LIM>
void launch_vl3d(const Fused3Launch& f, int parity, const FusedTile3* tiles, int nt) {
  constexpr size_t sm = fused3::Lay<ORDER>::bytes;
  static bool attrs = false;
  if (!attrs) {
    cudaFuncSetAttribute(fused3::k_vl3d<ORDER, RS, LIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attrs = true;
  }
  if (nt < 1) return;
  fused3::k_vl3d<ORDER, RS, LIM><<<nt, fused3::NT, sm, f.stream>>>(f.insts, tiles, parity, f.charact_proj,
                                                                   ORDER ? f.wsmaps : nullptr);
}

template <int RS>
void launch_pred_corr3(const Fused3Launch& f, int parity) {
  if (f.events) cudaEventRecord(f.events[1], f.stream);
  launch_vl3d<0, RS, dev::LIM_VL>(f, parity, f.tilesA, f.ntA);
  if (f.events) cudaEventRecord(f.events[2], f.stream);
  if (f.limiter == dev::LIM_MC) launch_vl3d<1, RS, dev::LIM_MC>(f, parity, f.tilesB, f.ntB);
  else if (f.limiter == dev::LIM_MM) launch_vl3d<1, RS, dev::LIM_MM>(f, parity, f.tilesB, f.ntB);
  else launch_vl3d<1, RS, dev::LIM_VL>(f, parity, f.tilesB, f.ntB);
  if (f.events) cudaEventRecord(f.events[3], f.stream);
}

}  // namespace

int fused3_step(const Fused3Launch& f, int parity) {
  if (f.events) cudaEventRecord(f.events[0], f.stream);
  fused::k_dt_batch<<<(f.ninst + 127) / 128, 128, 0, f.stream>>>(f.insts, f.ninst, parity, f.cour, f.dt_mode,
                                                                  f.dt_fixed, (unsigned*)nullptr);
  switch (f.rsolver) {
    case dev::RS_HLLD: launch_pred_corr3<dev::RS_HLLD>(f, parity); break;
    case dev::RS_HLLT: launch_pred_corr3<dev::RS_HLLT>(f, parity); break;
    default: launch_pred_corr3<dev::RS_HLL>(f, parity); break;
  }
  return 3;
}

int fused3_time(const Fused3Launch& f) {
  fused::k_time_batch<<<(f.ninst + 127) / 128, 128, 0, f.stream>>>(f.insts, f.ninst);
  return 1;
}

int fused3_cds(const Fused3Launch& f, int parity) {
  if (f.ntB > 0) fused3::k_cds3<<<f.ntB, 256, 0, f.stream>>>(f.insts, f.tilesB, parity);
  return 1;
}

// --- discrete adjoint of one fused 2D step ------------------------------

namespace {
// One reverse stage: S1 cells (unless the previous stage's gather ran it),
// S2 corners, S3 faces, S4 gather (optionally with the next stage's S1).
template <int RS>
void adj_stage(const FusedInst& I, const adjk::StageArgs& a, int lim, cudaStream_t st, bool run_cells,
               const adjk::StageArgs* next) {
  const int T = 128;
  const adjk::Box& R = a.R;
  const long long ncell = (long long)(R.ib - R.ia + 1) * (R.jb - R.ja + 1);
  const long long ncorner = (long long)(R.ib - R.ia + 2) * (R.jb - R.ja + 2);
  const long long nfx = (long long)(R.ib - R.ia + 2) * (R.jb - R.ja + 3);
  const long long nfy = (long long)(R.ib - R.ia + 3) * (R.jb - R.ja + 2);
  const int h = a.order == 0 ? 1 : 2;
  const long long ngat = (long long)(R.ib - R.ia + 1 + 2 * h) * (R.jb - R.ja + 1 + 2 * h);
  if (run_cells) adjk::k_cells<<<nblocks(ncell, T), T, 0, st>>>(I, a);
  adjk::k_corners<<<nblocks(ncorner, T), T, 0, st>>>(I, a);
  if (a.order == 0) adjk::k_faces<0, RS, false><<<nblocks(nfx + nfy, T), T, 0, st>>>(I, a, lim);
  else if (a.charact) adjk::k_faces<1, RS, true><<<nblocks(nfx + nfy, T), T, 0, st>>>(I, a, lim);
  else adjk::k_faces<1, RS, false><<<nblocks(nfx + nfy, T), T, 0, st>>>(I, a, lim);
  adjk::k_gather<<<nblocks(ngat, T), T, 0, st>>>(I, a, next ? *next : a, next ? 1 : 0);
}

void adj_fold(const FusedInst& I, double* Vw, double* Vb, cudaStream_t st) {
  const long long rx = I.nx - I.N[0] + 1, ry = I.ny - I.N[1] + 1;  // remappable positions per line
  const long long n = 12LL * (ry * I.nx + (I.ny - ry) * rx);
  adjk::k_fold2d<<<nblocks(n, 128), 128, 0, st>>>(I, Vw, Vb);
}
}  // namespace

int adj_step(const FusedInst& I, const AdjStep& s) {
  int launches = 0;
  cudaMemsetAsync(s.Vw, 0, 9 * (size_t)I.sv * sizeof(double), s.stream);
  cudaMemsetAsync(s.Vb, 0, 3 * (size_t)I.sv * sizeof(double), s.stream);
  // Bsb: the corrector's faces set the same range every step and the rest stays
  // zero, so the caller clears it once per reverse pass (clear_bsb on the first)
  if (s.clear_bsb) cudaMemsetAsync(s.Bsb, 0, 3 * (size_t)I.sv * sizeof(double), s.stream);
  if (s.fold_in) {
    adj_fold(I, s.G1w, s.G1b, s.stream);
    launches += 1;
  }
  adjk::StageArgs a;
  // corrector: order 1 on the active cells
  a.order = 1;
  a.charact = s.charact;
  a.dt = s.dt;
  a.R = {I.ng, I.ng + I.N[0] - 1, I.ng, I.ng + I.N[1] - 1};
  a.Wout = s.W1;
  a.Gw = s.G1w;
  a.Gb = s.G1b;
  a.Wsrc = s.Ws;
  a.Bsrc = s.Bs;
  a.Wn = s.Wn;
  a.Vw = s.Vw;
  a.Vb = s.Vb;
  a.Wsrc_b = s.Wsb;
  a.Bsrc_b = s.Bsb;
  a.Ub = s.Ub;
  a.Eb = s.Eb;
  a.Q = s.Q;
  // predictor: order 0 on cells 1..Ntot-2, half step
  adjk::StageArgs a0 = a;
  a0.order = 0;
  a0.charact = 0;
  a0.dt = 0.5 * s.dt;
  a0.R = {1, I.nx - 2, 1, I.ny - 2};
  a0.Wout = s.Ws;
  a0.Gw = s.Wsb;
  a0.Gb = s.Bsb;
  a0.Wsrc = s.Wn;
  a0.Bsrc = s.Bn;
  a0.Wsrc_b = s.Vw;
  a0.Bsrc_b = s.Vb;
  // the corrector's gather covers exactly the predictor's range: it runs the
  // predictor's S1 on the spot
  if (s.rsolver == dev::RS_HLLD) {
    adj_stage<dev::RS_HLLD>(I, a, s.limiter, s.stream, true, &a0);
    adj_stage<dev::RS_HLLD>(I, a0, s.limiter, s.stream, false, nullptr);
  } else if (s.rsolver == dev::RS_HLLT) {
    adj_stage<dev::RS_HLLT>(I, a, s.limiter, s.stream, true, &a0);
    adj_stage<dev::RS_HLLT>(I, a0, s.limiter, s.stream, false, nullptr);
  } else {
    adj_stage<dev::RS_HLL>(I, a, s.limiter, s.stream, true, &a0);
    adj_stage<dev::RS_HLL>(I, a0, s.limiter, s.stream, false, nullptr);
  }
  adj_fold(I, s.Vw, s.Vb, s.stream);
  return launches + 4 + 3 + 1;  // corrector stage, predictor stage without S1, the output fold
}

}  // namespace BNZ_NS
