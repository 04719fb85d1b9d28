// bnz_io.cu -- device side of the simulation's output: the history
// diagnostics as a device reduction, and state snapshots copied to the host
// while stepping continues.
//
// History (src/io/output.pyx:20-140 get_hst_vars_grid, MFIELD build): over the
// active cells of u = prim2cons(w) (bitwise the cons array the reference keeps
// between steps) the means of rho, E_kin = |m|^2 / (2 rho), E_th = E - E_kin -
// E_mag, E_mag = |B|^2 / 2, E, mx, my, mz, Bx, By, Bz, and rms(B_d) =
// sqrt(|<B_d^2> - <B_d>^2|).  Block partial sums then one final block: the
// result does not depend on scheduling.
//
// Snapshot: the current state (ghosts filled, cons derived) is copied on the
// context's stream into a snapshot buffer, then to caller-owned host memory on
// a copy stream, so the next steps run while the copy drains.
#include <cmath>
#include <string>

#include "bnz_ctx_internal.h"

using namespace bnzi;

namespace {

constexpr int NHS = 14;       // summed history quantities
constexpr int HIST_T = 256;
constexpr int HIST_BLOCKS = 148 * 4;

__global__ void k_hist_partial(GridDev g, const double* __restrict__ w, double* __restrict__ part) {
  __shared__ double red[HIST_T / 32][NHS];
  double acc[NHS];
#pragma unroll
  for (int q = 0; q < NHS; ++q) acc[q] = 0.;
  const int nx = g.i2 - g.i1 + 1, ny = g.j2 - g.j1 + 1, nz = g.k2 - g.k1 + 1;
  const long long n = (long long)nx * ny * nz;
  const double gamm1i = 1. / (g.gam - 1.);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = g.i1 + (int)(t % nx);
    const int j = g.j1 + (int)((t / nx) % ny);
    const int k = g.k1 + (int)(t / ((long long)nx * ny));
    const long long c = ((long long)k * g.ny + j) * g.nx + i;
    const double rho = w[c], vx = w[g.sv + c], vy = w[2 * g.sv + c], vz = w[3 * g.sv + c];
    const double pr = w[4 * g.sv + c];
    const double bx = w[6 * g.sv + c], by = w[7 * g.sv + c], bz = w[8 * g.sv + c];
    // prim2cons (eos_c.h:60-95)
    const double mx = rho * vx, my = rho * vy, mz = rho * vz;
    const double v2 = vx * vx + vy * vy + vz * vz;
    const double bx2 = bx * bx, by2 = by * by, bz2 = bz * bz;
    const double en = 0.5 * (rho * v2 + (bx2 + by2 + bz2)) + pr * gamm1i;
    // output.pyx:70-118
    const double rhoi = 1. / rho;
    const double ek = 0.5 * rhoi * (mx * mx + my * my + mz * mz);
    const double em = 0.5 * (bx2 + by2 + bz2);
    const double et = en - ek - em;
    const double v[NHS] = {rho, ek, et, em, en, mx, my, mz, bx, by, bz, bx2, by2, bz2};
#pragma unroll
    for (int q = 0; q < NHS; ++q) acc[q] += v[q];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NHS; ++q) {
    double x = acc[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[wid][q] = x;
  }
  __syncthreads();
  if (threadIdx.x < NHS) {
    double x = 0.;
    for (int q = 0; q < HIST_T / 32; ++q) x += red[q][threadIdx.x];
    part[(long long)blockIdx.x * NHS + threadIdx.x] = x;
  }
}

__global__ void k_hist_final(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  if (threadIdx.x < NHS) {
    double x = 0.;
    for (int b = 0; b < nblk; ++b) x += part[(long long)b * NHS + threadIdx.x];
    out[threadIdx.x] = x;
  }
}

// Face divergence of B over the active cells, the quantity constrained
// transport keeps at round-off (ct.pyx:15-91 updates each face by the curl of
// the edge EMFs, so sum over a cell's faces of A * dB cancels):
// div = sum_d (b_d[upper face] - b_d[lower face]) / dlf_d.  out[0] receives
// max |div| * dlf_x of the cell, out[1] max |B| of the cell-centred field, as
// the bit patterns of non-negative doubles (which order like the values).
__global__ void k_divb(GridDev g, const double* __restrict__ w, const double* __restrict__ b,
                       unsigned long long* __restrict__ out) {
  const int nx = g.i2 - g.i1 + 1, ny = g.j2 - g.j1 + 1, nz = g.k2 - g.k1 + 1;
  const long long n = (long long)nx * ny * nz;
  const long long sy = g.nx, sz = (long long)g.nx * g.ny;
  double dmax = 0., bmax = 0.;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = g.i1 + (int)(t % nx);
    const int j = g.j1 + (int)((t / nx) % ny);
    const int k = g.k1 + (int)(t / ((long long)nx * ny));
    const long long c = k * sz + j * sy + i;
    double d = (b[c + 1] - b[c]) * g.dlf_inv[0][i];
    if (g.dims >= 2) d += (b[g.sv + c + sy] - b[g.sv + c]) * g.dlf_inv[1][j];
    if (g.dims >= 3) d += (b[2 * g.sv + c + sz] - b[2 * g.sv + c]) * g.dlf_inv[2][k];
    dmax = fmax(dmax, fabs(d) * g.dlf[0][i]);
    const double bx = w[6 * g.sv + c], by = w[7 * g.sv + c], bz = w[8 * g.sv + c];
    bmax = fmax(bmax, sqrt(bx * bx + by * by + bz * bz));
  }
  for (int o = 16; o > 0; o >>= 1) {
    dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(dmax));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(bmax));
  }
}

}  // namespace

struct bnz_io {
  double* part = nullptr;   // HIST_BLOCKS x NHS partial sums, then NHS totals
  double* h_sums = nullptr; // pinned
  double* snap = nullptr;   // 21 fields: prim, cons, bfld
  cudaStream_t copy = nullptr;
  cudaEvent_t ready = nullptr, done = nullptr;
  bool pending = false;
};

namespace {

int io_init(bnz_ctx* c) {
  if (c->io) return BNZ_OK;
  bnz_io* o = new bnz_io();
  c->io = o;
  CKC(cudaMalloc((void**)&o->part, (HIST_BLOCKS + 1) * NHS * sizeof(double)));
  CKC(cudaMallocHost((void**)&o->h_sums, NHS * sizeof(double)));
  CKC(cudaStreamCreateWithFlags(&o->copy, cudaStreamNonBlocking));
  CKC(cudaEventCreateWithFlags(&o->ready, cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&o->done, cudaEventDisableTiming));
  return BNZ_OK;
}

}  // namespace

namespace bnzi {
void io_free(bnz_ctx* c) {
  if (!c || !c->io) return;
  bnz_io* o = c->io;
  if (o->copy) cudaStreamSynchronize(o->copy);
  if (o->part) cudaFree(o->part);
  if (o->h_sums) cudaFreeHost(o->h_sums);
  if (o->snap) cudaFree(o->snap);
  if (o->ready) cudaEventDestroy(o->ready);
  if (o->done) cudaEventDestroy(o->done);
  if (o->copy) cudaStreamDestroy(o->copy);
  delete o;
  c->io = nullptr;
}
}  // namespace bnzi

extern "C" {

int bnz_history(bnz_ctx* c, double* out) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (!out) return fail(c, BNZ_ERR_ARG, "null output");
  int rc = io_init(c);
  if (rc) return rc;
  bnz_io* o = c->io;
  StepArgs a = step_args(c);
  k_hist_partial<<<HIST_BLOCKS, HIST_T, 0, c->stream>>>(a.g, c->prim, o->part);
  k_hist_final<<<1, 32, 0, c->stream>>>(o->part, HIST_BLOCKS, o->part + HIST_BLOCKS * NHS);
  c->launches += 2;
  CKC(cudaGetLastError());
  CKC(cudaMemcpyAsync(o->h_sums, o->part + HIST_BLOCKS * NHS, NHS * sizeof(double), cudaMemcpyDeviceToHost,
                      c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  double t = 0., dt = 0.;
  long st = 0;
  rc = bnz_get_time(c, &t, &st, &dt);
  if (rc) return rc;
  const double ncells = (double)(c->i2 - c->i1 + 1) * (c->j2 - c->j1 + 1) * (c->k2 - c->k1 + 1);
  out[0] = (double)st;
  out[1] = t;
  for (int q = 0; q < NHS; ++q) out[2 + q] = o->h_sums[q] / ncells;
  // output.pyx:136-138
  for (int q = 13; q < 16; ++q) out[q] = std::sqrt(std::fabs(out[q] - out[q - 3] * out[q - 3]));
  return BNZ_OK;
}

int bnz_div_b(bnz_ctx* c, double* out) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (!out) return fail(c, BNZ_ERR_ARG, "null output");
  int rc = io_init(c);
  if (rc) return rc;
  bnz_io* o = c->io;
  StepArgs a = step_args(c);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(o->part);
  CKC(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), c->stream));
  k_divb<<<HIST_BLOCKS, HIST_T, 0, c->stream>>>(a.g, c->prim, c->bfld, d);
  c->launches += 1;
  CKC(cudaGetLastError());
  CKC(cudaMemcpyAsync(o->h_sums, d, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CKC(cudaStreamSynchronize(c->stream));
  out[0] = o->h_sums[0];
  out[1] = o->h_sums[1];
  return BNZ_OK;
}

int bnz_snapshot(bnz_ctx* c, double* prim, double* cons, double* bfld) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  int rc = io_init(c);
  if (rc) return rc;
  bnz_io* o = c->io;
  if (o->pending) CKC(cudaEventSynchronize(o->done));
  const size_t n = c->ncell;
  if (!o->snap) CKC(cudaMalloc((void**)&o->snap, 21 * n * sizeof(double)));
  rc = ensure_ghosts(c);
  if (rc) return rc;
  CKC(cudaMemcpyAsync(o->snap, c->prim, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CKC(cudaMemcpyAsync(o->snap + 9 * n, c->cons, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CKC(cudaMemcpyAsync(o->snap + 18 * n, c->bfld, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CKC(cudaEventRecord(o->ready, c->stream));
  CKC(cudaStreamWaitEvent(o->copy, o->ready, 0));
  if (prim) CKC(cudaMemcpyAsync(prim, o->snap, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, o->copy));
  if (cons) CKC(cudaMemcpyAsync(cons, o->snap + 9 * n, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, o->copy));
  if (bfld) CKC(cudaMemcpyAsync(bfld, o->snap + 18 * n, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, o->copy));
  CKC(cudaEventRecord(o->done, o->copy));
  o->pending = true;
  return BNZ_OK;
}

int bnz_snapshot_wait(bnz_ctx* c) {
  if (!c) return BNZ_ERR_ARG;
  if (!c->io || !c->io->pending) return BNZ_OK;
  CKC(cudaEventSynchronize(c->io->done));
  c->io->pending = false;
  return BNZ_OK;
}

}  // extern "C"
