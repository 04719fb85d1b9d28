// bnz_adjoint.cu -- host side of the adjoint entry points of include/bnz_gpu.h:
// fixed-dt rollouts recorded with checkpoints, their reverse pass, one-step
// VJPs and device-pointer state copies (for the torch.autograd wrapper).
//
// Tape of a rollout of nsteps steps with a checkpoint every K steps:
//   ckpt   the input state (w 9 + b 3 fields) of steps 0, K, 2K, ...
//   slot   two sets of K+1 records of one segment: the state w, b of each step
//          and its predictor output ws, bs.  The forward pass fills the last
//          segment's set directly; the reverse pass rebuilds every other
//          segment from its checkpoint.
//   work   two cotangent buffers (ping-pong, 12 fields each), the reverse
//          step's scratch (Wsb 9, Bsb 3, Ub 9, Eb 1, Q 72 fields) and a copy
//          of the final state (12)
// Memory: (12 ceil(nsteps/K) + 48 (K+1) + 142) fields of Ntot cells.
//
// The reverse pass runs on its own stream: while segment s is reversed there,
// segment s-1 is recomputed on the context's stream into the other slot set
// (events order the two).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bnz_ctx_internal.h"

using namespace bnzi;

struct bnz_adj {
  int nsteps = 0, K = 0, nck = 0;
  double dt = 0.;
  bool recorded = false;
  double* ckpt = nullptr;
  double* slot = nullptr;
  double* work = nullptr;
  size_t ckpt_cap = 0, slot_cap = 0, work_cap = 0;
  cudaStream_t rev = nullptr;         // reverse-pass stream
  cudaEvent_t ev_rec[2] = {nullptr, nullptr};  // slot set p rebuilt
  cudaEvent_t ev_rev[2] = {nullptr, nullptr};  // slot set p consumed
  cudaEvent_t ev_in = nullptr;
};

namespace {

constexpr int NW = 12;     // fields of a state record (9 prim + 3 face)
constexpr int NSLOT = 24;  // fields of a segment slot (w, b, ws, bs)
constexpr int NWORK = 2 * NW + 9 + 3 + 9 + 1 + 72 + NW;

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
  if (c->md.path != BNZ_PATH_FUSED || c->gd.dims != 2)
    return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint is built for the fused 2D path (path = fused, dims = 2)");
  if (c->md.kappa0 > 0.) return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint covers the hyperbolic step only (kappa0 = 0)");
  if (c->md.rsolver != BNZ_RS_HLL && c->md.rsolver != BNZ_RS_HLLD && c->md.rsolver != BNZ_RS_HLLT)
    return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint is built for rsolver hll, hllt and hlld");
  // constant gravity is differentiated; the driving force is a random field
  // advanced every step, which the tape does not keep
  if (drive_on(c->md)) return fail(c, BNZ_ERR_UNSUPPORTED, "the adjoint is built without turbulence driving");
  if (!c->adj) c->adj = new bnz_adj();
  bnz_adj* A = c->adj;
  if (!A->rev) {
    // the reverse steps are the critical path: their stream outranks the
    // context's stream, on which the previous segment is recomputed meanwhile
    int least = 0, greatest = 0;
    CKC(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CKC(cudaStreamCreateWithPriority(&A->rev, cudaStreamNonBlocking, greatest));
    for (int p = 0; p < 2; ++p) {
      CKC(cudaEventCreateWithFlags(&A->ev_rec[p], cudaEventDisableTiming));
      CKC(cudaEventCreateWithFlags(&A->ev_rev[p], cudaEventDisableTiming));
    }
    CKC(cudaEventCreateWithFlags(&A->ev_in, cudaEventDisableTiming));
  }
  return BNZ_OK;
}

double* field(double* base, bnz_ctx* c, size_t k) { return base + k * c->ncell; }

// slot q of slot set p
double* slot_at(bnz_ctx* c, int p, int q) { return field(c->adj->slot, c, ((size_t)p * (c->adj->K + 1) + q) * NSLOT); }

// copy a 12-field state record (w then b) on stream st
int copy_state(bnz_ctx* c, double* dw, double* db, const double* sw, const double* sb, cudaStream_t st) {
  CKC(cudaMemcpyAsync(dw, sw, 9 * c->ncell * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CKC(cudaMemcpyAsync(db, sb, 3 * c->ncell * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return BNZ_OK;
}

// one forward step of fixed dt from the context's state (on its stream),
// recording its input state and predictor output into slot q of set p (and,
// when last, the output state into slot q + 1)
int record_step(bnz_ctx* c, double dt, int p, int q, bool last) {
  double* s = slot_at(c, p, q);
  int rc = copy_state(c, s, s + 9 * c->ncell, c->prim, c->bfld, c->stream);
  if (rc) return rc;
  c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
  rc = step_impl(c, dt);
  if (rc) return rc;
  rc = copy_state(c, s + 12 * c->ncell, s + 21 * c->ncell, c->cons_s, c->bfld_s, c->stream);
  if (rc) return rc;
  if (last) {
    double* s1 = slot_at(c, p, q + 1);
    rc = copy_state(c, s1, s1 + 9 * c->ncell, c->prim, c->bfld, c->stream);
  }
  return rc;
}

// rebuild segment seg of the recorded rollout into slot set p (context stream)
int recompute_segment(bnz_ctx* c, int seg, int p) {
  bnz_adj* A = c->adj;
  const int n0 = seg * A->K;
  const int m = (A->nsteps - n0) < A->K ? (A->nsteps - n0) : A->K;
  double* ck = field(A->ckpt, c, (size_t)seg * NW);
  int rc = copy_state(c, c->prim, c->bfld, ck, ck + 9 * c->ncell, c->stream);
  if (rc) return rc;
  for (int q = 0; q < m; ++q) {
    rc = record_step(c, A->dt, p, q, q == m - 1);
    if (rc) return rc;
  }
  return BNZ_OK;
}

// reverse step of slot q of set p on stream st: cotangent (gw, gb) of the step's
// output -> (vw, vb); fold_in: gw, gb may carry ghost entries
int reverse_step(bnz_ctx* c, double dt, int p, int q, double* gw, double* gb, double* vw, double* vb, bool fold_in,
                 cudaStream_t st) {
  bnz_adj* A = c->adj;
  double* s = slot_at(c, p, q);
  double* s1 = slot_at(c, p, q + 1);
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
  a.charact = c->md.charact_proj ? 1 : 0;
  a.fold_in = fold_in ? 1 : 0;
  a.clear_bsb = fold_in ? 1 : 0;  // the first reverse step of a pass
  a.stream = st;
  c->launches += c->L->adj_step(make_inst(c), a);
  CKC(cudaGetLastError());
  return BNZ_OK;
}

double* keep_at(bnz_ctx* c) { return field(c->adj->work, c, NWORK - NW); }

}  // namespace

namespace bnzi {
void adj_free(bnz_ctx* c) {
  if (!c || !c->adj) return;
  bnz_adj* A = c->adj;
  if (A->rev) cudaStreamSynchronize(A->rev);
  if (A->ckpt) cudaFree(A->ckpt);
  if (A->slot) cudaFree(A->slot);
  if (A->work) cudaFree(A->work);
  for (int p = 0; p < 2; ++p) {
    if (A->ev_rec[p]) cudaEventDestroy(A->ev_rec[p]);
    if (A->ev_rev[p]) cudaEventDestroy(A->ev_rev[p]);
  }
  if (A->ev_in) cudaEventDestroy(A->ev_in);
  if (A->rev) cudaStreamDestroy(A->rev);
  delete A;
  c->adj = nullptr;
}
}  // namespace bnzi

extern "C" {

int bnz_set_state_device(bnz_ctx* c, const double* prim, const double* bfld) {
  if (!c || !c->prim) return fail(c, BNZ_ERR_ARG, "context not created");
  if (!prim || !bfld) return fail(c, BNZ_ERR_ARG, "null state pointer");
  int rc = copy_state(c, c->prim, c->bfld, prim, bfld, c->stream);
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
  A->K = K;
  rc = ensure_buf(c, &A->ckpt, &A->ckpt_cap, (size_t)NW * nck);
  if (rc) return rc;
  rc = ensure_buf(c, &A->slot, &A->slot_cap, (size_t)NSLOT * 2 * (K + 1));
  if (rc) return rc;
  // the previous reverse pass may still read the slots
  CKC(cudaStreamSynchronize(A->rev));
  const int last = nck - 1, n_last = last * K;
  for (int n = 0; n < nsteps; ++n) {
    if (n % K == 0) {
      double* ck = field(A->ckpt, c, (size_t)(n / K) * NW);
      rc = copy_state(c, ck, ck + 9 * c->ncell, c->prim, c->bfld, c->stream);
      if (rc) return rc;
    }
    if (n >= n_last) {
      // the last segment is recorded as it runs: the reverse pass starts there
      rc = record_step(c, dt, last & 1, n - n_last, n == nsteps - 1);
    } else {
      c->launches += c->L->set_dt(c->stream, c->d_ds, dt);
      rc = step_impl(c, dt);
    }
    if (rc) return rc;
  }
  A->nsteps = nsteps;
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
  rc = ensure_buf(c, &A->work, &A->work_cap, NWORK);
  if (rc) return rc;
  cudaStream_t S1 = c->stream, S2 = A->rev;
  // keep the final state: recomputing segments moves the context's state
  double* keep = keep_at(c);
  rc = copy_state(c, keep, keep + 9 * c->ncell, c->prim, c->bfld, S1);
  if (rc) return rc;
  double* G = field(A->work, c, 0);
  double* V = field(A->work, c, NW);
  rc = copy_state(c, G, G + 9 * c->ncell, gprim, gbfld, S1);
  if (rc) return rc;
  CKC(cudaEventRecord(A->ev_in, S1));
  CKC(cudaStreamWaitEvent(S2, A->ev_in, 0));
  // the last segment's slots were filled by the forward pass
  for (int seg = A->nck - 1; seg >= 0; --seg) {
    const int p = seg & 1;
    const int m = (A->nsteps - seg * A->K) < A->K ? (A->nsteps - seg * A->K) : A->K;
    if (seg >= 1) {
      // rebuild the previous segment into the other set once segment seg+1
      // (the last user of that set) has been reversed
      if (seg + 1 <= A->nck - 1) CKC(cudaStreamWaitEvent(S1, A->ev_rev[p ^ 1], 0));
      rc = recompute_segment(c, seg - 1, p ^ 1);
      if (rc) return rc;
      CKC(cudaEventRecord(A->ev_rec[p ^ 1], S1));
    }
    for (int q = m - 1; q >= 0; --q) {
      const bool first = seg == A->nck - 1 && q == m - 1;
      rc = reverse_step(c, A->dt, p, q, G, G + 9 * c->ncell, V, V + 9 * c->ncell, first, S2);
      if (rc) return rc;
      double* t = G;
      G = V;
      V = t;
    }
    CKC(cudaEventRecord(A->ev_rev[p], S2));
    if (seg >= 1) CKC(cudaStreamWaitEvent(S2, A->ev_rec[p ^ 1], 0));
  }
  CKC(cudaStreamWaitEvent(S1, A->ev_rev[0], 0));
  rc = copy_state(c, gprim0, gbfld0, G, G + 9 * c->ncell, S1);
  if (rc) return rc;
  rc = copy_state(c, c->prim, c->bfld, keep, keep + 9 * c->ncell, S1);
  if (rc) return rc;
  c->ghosts_stale = true;
  rc = refresh_cds(c);
  if (rc) return rc;
  // the slots now hold segment 0: a second reverse pass needs a new forward
  A->recorded = false;
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
  CKC(cudaStreamSynchronize(A->rev));
  A->K = 1;
  rc = ensure_buf(c, &A->slot, &A->slot_cap, (size_t)NSLOT * 2 * 2);
  if (rc) return rc;
  rc = ensure_buf(c, &A->work, &A->work_cap, NWORK);
  if (rc) return rc;
  rc = copy_state(c, c->prim, c->bfld, prim, bfld, c->stream);
  if (rc) return rc;
  rc = record_step(c, dt, 0, 0, true);
  if (rc) return rc;
  double* G = field(A->work, c, 0);
  double* V = field(A->work, c, NW);
  rc = copy_state(c, G, G + 9 * c->ncell, gprim1, gbfld1, c->stream);
  if (rc) return rc;
  rc = reverse_step(c, dt, 0, 0, G, G + 9 * c->ncell, V, V + 9 * c->ncell, true, c->stream);
  if (rc) return rc;
  rc = copy_state(c, gprim0, gbfld0, V, V + 9 * c->ncell, c->stream);
  if (rc) return rc;
  c->ghosts_stale = true;
  rc = refresh_cds(c);
  if (rc) return rc;
  CKC(cudaGetLastError());
  return BNZ_OK;
}

}  // extern "C"
