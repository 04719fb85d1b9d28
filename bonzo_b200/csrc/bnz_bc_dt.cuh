// bnz_bc_dt.cuh -- ghost fill, CFL time step and time bookkeeping kernels.
// Included inside the per-floating-point-mode namespace.
#pragma once

namespace bcdt {

using namespace dev;

struct FieldList {
  int n;
  int f[12];  // 0..8 prim variable, 9..11 face component
};

// Source index along the BC axis for ghost index `d` (util_bc.pyx:9-251,
// grid_bc_funcs.pyx:36-330).  Returns 0 = no write, 1 = copy src*sgn,
// 2 = write zero.
__device__ __forceinline__ int bc_map(int flag, int side, int d, int a1, int a2, int ng, bool normal_cell,
                                      bool face_normal, int face_aware, int& src, double& sgn) {
  sgn = 1.;
  if (flag == 0) {  // periodic
    src = side == 0 ? d + (a2 - a1 + 1) : d - (a2 - a1 + 1);
    return 1;
  }
  if (flag == 1) {  // outflow (prolong); face-aware keeps the CT face a2+1
    if (side == 0) { src = a1; return 1; }
    if (face_normal && face_aware) {
      if (d == a2 + 1) return 0;
      src = a2 + 1;
      return 1;
    }
    src = a2;
    return 1;
  }
  // reflect
  if (face_normal) {
    if (side == 1 && d == a2 + 1) return 2;
    src = side == 0 ? 2 * a1 - d : 2 * a2 + 2 - d;
    sgn = -1.;
    return 1;
  }
  src = side == 0 ? 2 * a1 - 1 - d : 2 * a2 + 1 - d;
  sgn = normal_cell ? -1. : 1.;
  return 1;
}

// Ghost fill along one axis for a list of fields, both sides at once
// (grid_bc.pyx:612-623 calls z, then y, then x; the host launches in that
// order so corners come out as in the reference).
__global__ void k_bc_axis(GridDev g, int ax, double* prim, double* bfld, FieldList fl, int flag0, int flag1,
                          int face_aware) {
  const int ng = g.ng;
  const int N[3] = {g.nx, g.ny, g.nz};
  const int a1 = ax == 0 ? g.i1 : ax == 1 ? g.j1 : g.k1;
  const int a2 = ax == 0 ? g.i2 : ax == 1 ? g.j2 : g.k2;
  const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;  // the two other axes
  const long long nother = (long long)N[o1] * N[o2];
  const long long per_field = 2LL * ng * nother;
  const int fi = blockIdx.y;
  if (fi >= fl.n) return;
  const int f = fl.f[fi];
  double* A = f < NM ? prim + (long long)f * g.sv : bfld + (long long)(f - NM) * g.sv;
  const bool face_normal = (f >= NM) && (f - NM == ax);
  const bool normal_cell = (f == VX + ax) || (f == BX + ax);
  const long long st[3] = {1, g.nx, (long long)g.nx * g.ny};
  // along x the ghost layers of a row are neighbours in memory: the layer is
  // the fastest index there, so that a warp reads and writes a few rows'
  // ends instead of one double per row
  const long long nl = 2LL * ng;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per_field;
       t += (long long)gridDim.x * blockDim.x) {
    long long rest = ax == 0 ? t / nl : t % nother;
    int layer = (int)(ax == 0 ? t % nl : t / nother);
    int side = layer / ng, gl = layer % ng;
    int c1 = (int)(rest % N[o1]), c2 = (int)(rest / N[o1]);
    int d = side == 0 ? a1 - ng + gl : a2 + 1 + gl;
    int flag = side == 0 ? flag0 : flag1;
    int src;
    double sgn;
    int act = bc_map(flag, side, d, a1, a2, ng, normal_cell, face_normal, face_aware, src, sgn);
    long long base = c1 * st[o1] + c2 * st[o2];
    if (act == 1) A[base + d * st[ax]] = sgn * A[base + src * st[ax]];
    else if (act == 2) A[base + d * st[ax]] = 0.;
    // reflect zeroes the first active normal face as well (set_layer at a1)
    if (flag == 2 && face_normal && side == 0 && gl == 0) A[base + a1 * st[ax]] = 0.;
  }
}

// new_dt.pyx:55-99 + 117: per-cell (|v_d| + c_f)/dx_d, max over active cells.
// Non-negative doubles order like their bit patterns, so the global max is an
// integer atomicMax on the bits.
// hydro: the hydro build's sound speed (no magnetic field).
__global__ void k_cds_max(GridDev g, const double* __restrict__ w, unsigned long long* slot, int hydro) {
  double m = 0.;
  const int nxa = g.i2 - g.i1 + 1, nya = g.j2 - g.j1 + 1, nza = g.k2 - g.k1 + 1;
  const long long n = (long long)nxa * nya * nza;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = g.i1 + (int)(t % nxa);
    long long r = t / nxa;
    int j = g.j1 + (int)(r % nya), k = g.k1 + (int)(r / nya);
    long long c = ((long long)k * g.ny + j) * g.nx + i;
    double ww[NM];
#pragma unroll
    for (int q = 0; q < NM; ++q) ww[q] = w[q * g.sv + c];
    double vf = hydro ? fms_hydro(ww, g.gam) : fms(ww, g.gam);
    double cx = fabs(ww[VX]) + vf, cy = 0., cz = 0.;
    if (g.dims >= 2) cy = fabs(ww[VY]) + vf;
    if (g.dims >= 3) cz = fabs(ww[VZ]) + vf;
    double cds = fmax(fmax(cx / g.dlf[0][i], cy / g.dlf[1][j]), cz / g.dlf[2][k]);
    if (cds > m) m = cds;
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

__global__ void k_dt_reset(DtState* ds) { ds->cdsmax_bits = 0ULL; }

// new_dt.pyx:117 and vanleer.pyx:95-96: dt = cour/max, clipped to tmax.
__global__ void k_dt_finalize(DtState* ds, double cour, int clip) {
  double m = __longlong_as_double((long long)ds->cdsmax_bits);
  double dt = cour / m;
  if (clip && ds->time + dt > ds->tmax) dt = ds->tmax - ds->time;
  if (clip && ds->time >= ds->tmax) dt = 0.;
  ds->dt = dt;
}

__global__ void k_dt_set(DtState* ds, double dt) { ds->dt = dt; }

// the fixed time step (vanleer.pyx:87-99 with fixdt), zero once the record's
// time has reached tmax: the loop takes no further step
__global__ void k_dt_fixed(DtState* ds, double dt) { ds->dt = ds->time >= ds->tmax ? 0. : dt; }

// vanleer.pyx:166-167
__global__ void k_time_advance(DtState* ds) {
  if (ds->dt > 0.) {
    ds->time += ds->dt;
    ds->step += 1;
  }
}

}  // namespace bcdt
