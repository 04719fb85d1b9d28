// bnz_adjoint.cu -- host side of the adjoint entry points of include/bnz_gpu.h:
// fixed-dt rollouts recorded with checkpoints, their reverse pass, one-step
// VJPs and device-pointer state copies (for the torch.autograd wrapper).
//
// Tape of a rollout of nsteps steps with a checkpoint every K steps:
//   ckpt   the input state (w 9 + b 3 fields) of steps 0, K, 2K, ...
//   slot   K+1 records of one segment rebuilt during the reverse pass: the
//          state w, b of each step and its predictor output ws, bs
//   work   two cotangent buffers (ping-pong, 12 fields each) and the reverse
//          step's scratch (Wsb 9, Bsb 3, Ub 9, Eb 1, Q 72 fields)
// Memory: (12 ceil(nsteps/K) + 24 (K+1) + 118) fields of Ntot cells.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bnz_ctx_internal.h"

using namespace bnzi;

struct bnz_adj {
  int nsteps = 0, K = 0, nck = 0, nslot = 0;
  double dt = 0.;
  bool recorded = false;
  double* ckpt = nullptr;
  double* slot = nullptr;
  double* work = nullptr;
  size_t ckpt_cap = 0, slot_cap = 0, work_cap = 0;
};

namespace {

constexpr int NW = 12;     // fields of a state record (9 prim + 3 face)
constexpr int NSLOT = 24;  // fields of a segment slot (w, b, ws, bs)
constexpr int NWORK = 2 * NW + 9 + 3 + 9 + 1 + 72;

int ensure_buf(bnz_ctx* c, double** p, size_t* cap, size_t fields) {
  const size_t bytes = fields * c->ncell * sizeof(double);
  if (*cap >= bytes) return BNZ_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) return fail(c, BNZ_ERR_NOMEM, std::string("adjoint tape: ") + cudaGetErrorString(e));
  *cap = bytes;
  return BNZ_OK;
}

int check_adjoint_ctx(bnz_ctx* c) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (c->md.path != BNZ_PATH_FUSED)
    return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint is built for the fused 2D path (path = fused)");
  if (c->md.kappa0 > 0.) return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint covers the hyperbolic step only (kappa0 = 0)");
  if (c->md.rsolver != BNZ_RS_HLL && c->md.rsolver != BNZ_RS_HLLD)
    return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint is built for rsolver hll and hlld");
  if (!c->adj) c->adj = new bnz_adj();
  return BNZ_OK;
}

double* field(double* base, bnz_ctx* c, size_t k) { return base + k * c->ncell; }

// copy a 12-field state record (w then b) in or out of the context's state
int copy_state(bnz_ctx* c, double* dw, double* db, const double* sw, const double* sb) {
  CKC(cudaMemcpyAsync(dw, sw, 9 * c->ncell * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CKC(cudaMemcpyAsync(db, sb, 3 * c->ncell * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return BNZ_OK;
}

// one forward step of fixed dt from the context's state, recording its input
// state and predictor output into slot q (and the output state into q + 1)
int record_step(bnz_ctx* c, double dt, int q, bool last) {
  bnz_adj* A = c->adj;
  double* s = field(A->slot, c, (size_t)q * NSLOT);
  int rc = copy_state(c, s, s + 9 * c->ncell, c->prim, c->bfld);
  if (rc) return rc;
  c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
  rc = step_impl(c, dt);
  if (rc) return rc;
  rc = copy_state(c, s + 12 * c->ncell, s + 21 * c->ncell, c->cons_s, c->bfld_s);
  if (rc) return rc;
  if (last) {
    double* s1 = field(A->slot, c, (size_t)(q + 1) * NSLOT);
    rc = copy_state(c, s1, s1 + 9 * c->ncell, c->prim, c->bfld);
  }
  return rc;
}

// reverse step of slot q: cotangent (gw, gb) of slot q+1's state -> (vw, vb)
int reverse_step(bnz_ctx* c, double dt, int q, double* gw, double* gb, double* vw, double* vb) {
  bnz_adj* A = c->adj;
  double* s = field(A->slot, c, (size_t)q * NSLOT);
  double* s1 = field(A->slot, c, (size_t)(q + 1) * NSLOT);
  double* wk = field(A->work, c, 2 * NW);
  AdjStep a;
  a.Wn = s;
  a.Bn = s + 9 * c->ncell;
  a.Ws = s + 12 * c->ncell;
  a.Bs = s + 21 * c->ncell;
  a.W1 = s1;
  a.G1w = gw;
  a.G1b = gb;
  a.Vw = vw;
  a.Vb = vb;
  a.Wsb = wk;
  a.Bsb = wk + 9 * c->ncell;
  a.Ub = wk + 12 * c->ncell;
  a.Eb = wk + 21 * c->ncell;
  a.Q = wk + 22 * c->ncell;
  a.dt = dt;
  a.rsolver = c->md.rsolver;
  a.limiter = c->md.limiter;
  a.stream = c->stream;
  c->launches += c->L->adj_step(make_inst(c), a);
  CKC(cudaGetLastError());
  return BNZ_OK;
}

}  // namespace

namespace bnzi {
void adj_free(bnz_ctx* c) {
  if (!c || !c->adj) return;
  if (c->adj->ckpt) cudaFree(c->adj->ckpt);
  if (c->adj->slot) cudaFree(c->adj->slot);
  if (c->adj->work) cudaFree(c->adj->work);
  delete c->adj;
  c->adj = nullptr;
}
}  // namespace bnzi

extern "C" {

int bnz_set_state_device(bnz_ctx* c, const double* prim, const double* bfld) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (!prim || !bfld) return fail(c, BNZ_ERR_ARG, "null state pointer");
  int rc = copy_state(c, c->prim, c->bfld, prim, bfld);
  if (rc) return rc;
  StepArgs a = step_args(c);
  c->launches += c->L->prim2cons_all(a);
  c->ghosts_stale = false;
  rc = refresh_cds(c);
  if (rc) return rc;
  CKC(cudaGetLastError());
  return BNZ_OK;
}

int bnz_get_state_device(bnz_ctx* c, double* prim, double* bfld) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  int rc = ensure_ghosts(c);
  if (rc) return rc;
  if (prim) CKC(cudaMemcpyAsync(prim, c->prim, 9 * c->ncell * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (bfld) CKC(cudaMemcpyAsync(bfld, c->bfld, 3 * c->ncell * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return BNZ_OK;
}

int bnz_rollout_forward(bnz_ctx* c, int nsteps, double dt, int checkpoint_every) {
  int rc = check_adjoint_ctx(c);
  if (rc) return rc;
  if (nsteps < 1 || checkpoint_every < 1) return fail(c, BNZ_ERR_ARG, "nsteps and checkpoint_every must be >= 1");
  if (!(dt > 0.) || std::isinf(dt)) return fail(c, BNZ_ERR_ARG, "dt must be finite and > 0");
  bnz_adj* A = c->adj;
  A->recorded = false;
  const int K = checkpoint_every < nsteps ? checkpoint_every : nsteps;
  const int nck = (nsteps + K - 1) / K;
  rc = ensure_buf(c, &A->ckpt, &A->ckpt_cap, (size_t)NW * nck);
  if (rc) return rc;
  for (int n = 0; n < nsteps; ++n) {
    if (n % K == 0) {
      double* ck = field(A->ckpt, c, (size_t)(n / K) * NW);
      rc = copy_state(c, ck, ck + 9 * c->ncell, c->prim, c->bfld);
      if (rc) return rc;
    }
    c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
    rc = step_impl(c, dt);
    if (rc) return rc;
  }
  A->nsteps = nsteps;
  A->K = K;
  A->nck = nck;
  A->dt = dt;
  A->recorded = true;
  CKC(cudaGetLastError());
  return BNZ_OK;
}

int bnz_rollout_adjoint(bnz_ctx* c, const double* gprim, const double* gbfld, double* gprim0, double* gbfld0) {
  int rc = check_adjoint_ctx(c);
  if (rc) return rc;
  bnz_adj* A = c->adj;
  if (!A->recorded) return fail(c, BNZ_ERR_STATE, "no rollout recorded (bnz_rollout_forward first)");
  if (!gprim || !gbfld || !gprim0 || !gbfld0) return fail(c, BNZ_ERR_ARG, "null cotangent pointer");
  rc = ensure_buf(c, &A->slot, &A->slot_cap, (size_t)NSLOT * (A->K + 1));
  if (rc) return rc;
  rc = ensure_buf(c, &A->work, &A->work_cap, NWORK);
  if (rc) return rc;
  // keep the final state: the reverse pass rebuilds segments in the context
  double* keep = field(A->slot, c, (size_t)A->K * NSLOT + 12);
  rc = copy_state(c, keep, keep + 9 * c->ncell, c->prim, c->bfld);
  if (rc) return rc;
  double* G = field(A->work, c, 0);
  double* V = field(A->work, c, NW);
  rc = copy_state(c, G, G + 9 * c->ncell, gprim, gbfld);
  if (rc) return rc;
  for (int seg = A->nck - 1; seg >= 0; --seg) {
    const int n0 = seg * A->K;
    const int m = (A->nsteps - n0) < A->K ? (A->nsteps - n0) : A->K;
    double* ck = field(A->ckpt, c, (size_t)seg * NW);
    rc = copy_state(c, c->prim, c->bfld, ck, ck + 9 * c->ncell);
    if (rc) return rc;
    for (int q = 0; q < m; ++q) {
      rc = record_step(c, A->dt, q, q == m - 1);
      if (rc) return rc;
    }
    for (int q = m - 1; q >= 0; --q) {
      rc = reverse_step(c, A->dt, q, G, G + 9 * c->ncell, V, V + 9 * c->ncell);
      if (rc) return rc;
      double* t = G;
      G = V;
      V = t;
    }
  }
  rc = copy_state(c, gprim0, gbfld0, G, G + 9 * c->ncell);
  if (rc) return rc;
  rc = copy_state(c, c->prim, c->bfld, keep, keep + 9 * c->ncell);
  if (rc) return rc;
  c->ghosts_stale = true;
  rc = refresh_cds(c);
  if (rc) return rc;
  CKC(cudaGetLastError());
  return BNZ_OK;
}

int bnz_step_adjoint(bnz_ctx* c, double dt, const double* prim, const double* bfld, const double* gprim1,
                     const double* gbfld1, double* gprim0, double* gbfld0) {
  int rc = check_adjoint_ctx(c);
  if (rc) return rc;
  if (!(dt > 0.) || std::isinf(dt)) return fail(c, BNZ_ERR_ARG, "dt must be finite and > 0");
  if (!prim || !bfld || !gprim1 || !gbfld1 || !gprim0 || !gbfld0) return fail(c, BNZ_ERR_ARG, "null pointer");
  bnz_adj* A = c->adj;
  A->recorded = false;
  rc = ensure_buf(c, &A->slot, &A->slot_cap, (size_t)NSLOT * 2);
  if (rc) return rc;
  rc = ensure_buf(c, &A->work, &A->work_cap, NWORK);
  if (rc) return rc;
  rc = copy_state(c, c->prim, c->bfld, prim, bfld);
  if (rc) return rc;
  rc = record_step(c, dt, 0, true);
  if (rc) return rc;
  double* G = field(A->work, c, 0);
  double* V = field(A->work, c, NW);
  rc = copy_state(c, G, G + 9 * c->ncell, gprim1, gbfld1);
  if (rc) return rc;
  rc = reverse_step(c, dt, 0, G, G + 9 * c->ncell, V, V + 9 * c->ncell);
  if (rc) return rc;
  rc = copy_state(c, gprim0, gbfld0, V, V + 9 * c->ncell);
  if (rc) return rc;
  c->ghosts_stale = true;
  rc = refresh_cds(c);
  if (rc) return rc;
  CKC(cudaGetLastError());
  return BNZ_OK;
}

}  // extern "C"
