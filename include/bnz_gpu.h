/*
 * bnz_gpu.h -- C ABI of the B200 VL2 + HLLD + CT step (libbnzgpu.so).
 *
 * Drop-in boundary for the reference's integrator / grid calls
 * (sergekomarov/bonzo).  Plain C types only: integer status codes, opaque
 * contexts, double arrays in the reference's layout.
 *
 * Layout of every state array (the reference's GridData, src/coordinates/
 * grid.pyx:30-52): C-contiguous [var][k][j][i] over the FULL grid including
 * ghost cells, FP64.  prim / cons have 9 variables in the order
 * rho, vx|mx, vy|my, vz|mz, p|E, passive scalar, Bx, By, Bz (src/defs_c.h:68-85);
 * bfld has 3 face-centred components, bfld[0][k][j][i] on the x face at the
 * left edge of cell i (and likewise for y, z).
 *
 * Ownership: host pointers are borrowed for the duration of a call only.
 * Device buffers belong to the context.  Calls on one context are ordered on
 * its CUDA stream and are not re-entrant; one context per host thread.
 *
 * Every function returns BNZ_OK (0) or a positive bnz_status; the message of
 * the last failure is bnz_last_error(ctx).
 */
#ifndef BNZ_GPU_H
#define BNZ_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  BNZ_OK = 0,
  BNZ_ERR_ARG = 1,         /* bad argument or configuration (rejected before any launch) */
  BNZ_ERR_CUDA = 2,        /* CUDA runtime error */
  BNZ_ERR_STATE = 3,       /* non-physical state met on the device (rho<=0, p<=0, NaN) */
  BNZ_ERR_UNSUPPORTED = 4, /* option not available in this build */
  BNZ_ERR_TIMEOUT = 5,     /* a bounded device wait ran out */
  BNZ_ERR_NOMEM = 6
} bnz_status;

/* Method enums, values as the reference's integrator enums
 * (src/integration/integrator.pxd:52-91) where it has them. */
enum { BNZ_RS_HLL = 0, BNZ_RS_HLLC = 1, BNZ_RS_HLLD = 2, BNZ_RS_HLLT = 3 };
enum { BNZ_RCN_CONST = 0, BNZ_RCN_LINEAR = 1 };
enum { BNZ_LIM_VL = 0, BNZ_LIM_MC = 1, BNZ_LIM_MM = 2 };
enum { BNZ_BC_PERIODIC = 0, BNZ_BC_OUTFLOW = 1, BNZ_BC_REFLECT = 2 };
enum { BNZ_TC_ISO = 0, BNZ_TC_ANISO = 1 };
/* kernel path: fused tile kernels (default), one kernel per reference loop
 * (plain), or the plain path's decomposition with each face's flux formed once
 * from per-cell slopes and one fused update per stage (split).  All three
 * give the same bits in the exact build; hydro mode runs on plain or split. */
enum { BNZ_PATH_FUSED = 0, BNZ_PATH_PLAIN = 1, BNZ_PATH_SPLIT = 2 };

/* Grid: the [computation] Nx..Nz / xmin..zmax keys and the [physics]
 * bc_x1..bc_z2 flags (src/coordinates/grid.pyx:107-232,
 * src/bc/grid_bc.pyx:45-50).  dims replaces the reference's D2D/D3D build
 * flags. */
typedef struct {
  int Nx, Ny, Nz;
  int dims;
  double lmin[3], lmax[3];
  int bc[3][2];
} bnz_grid_desc;

/* Method: the [computation] / [physics] keys of the step
 * (src/integration/integrator.pyx:205-291, src/dissipation/diffusion.pyx:30-49).
 * limiter is the added `limiter: vl|mc|mm` key (the reference hard-wires vl).
 * outflow_face_aware keeps the CT-updated outer face under outflow BCs.
 * exact_fp selects kernels built without multiply-add contraction, which
 * reproduce the CPU reference bit for bit; path selects fused, plain or split kernels.
 * Source terms (src/srcterms, applied in both stages by
 * integrator.pyx:132-170 add_source_terms): grav = the [physics] gx, gy, gz
 * constant acceleration (gravity.pyx:17-19); drive_f0 / drive_tau / drive_nmod
 * = the [physics] f0, tau, nmod of the solenoidal driving force
 * (turb_driv.pyx:27-29), whose random mode amplitudes come from a splitmix64
 * stream seeded with drive_seed.  Zero f0 and grav switch them off.
 * hydro = 1 is the reference's hydro build (MFIELD 0, src/defs_c.h:72-96):
 * the field entries of prim / cons and the face field are held at zero, no CT
 * runs, signal speeds are the hydro sound speed, and rsolver is hll or hllc
 * (fluxes_c.c:175-223, 232-327); plain or split path, no charact_proj, no
 * conduction. */
typedef struct {
  double gam, cour;
  int rsolver, reconstr, limiter, charact_proj;
  double kappa0;
  int thcond_type, sat_hfe;
  double cour_diff;
  int fixdt;
  double dt_fixed;
  int outflow_face_aware;
  int exact_fp;
  int path;
  double grav[3];
  double drive_f0, drive_tau;
  int drive_nmod;
  unsigned long long drive_seed;
  int hydro;
} bnz_method_desc;

typedef struct bnz_ctx bnz_ctx;

/* BnzGrid(usr_dir) + BnzIntegr(gc, usr_dir): src/coordinates/grid.pyx:59-81,
 * src/integration/integrator.pyx:23-28.  Allocates the device state. */
int bnz_create(const bnz_grid_desc* grid, const bnz_method_desc* method, bnz_ctx** out);
int bnz_destroy(bnz_ctx* ctx);
const char* bnz_last_error(const bnz_ctx* ctx);
/* Ntot[3] (x, y, z, ghosts included) and the ghost width ng. */
int bnz_shape(const bnz_ctx* ctx, int* ntot, int* ng);

/* Upload a full state (the arrays set_problem writes; problem.pyx API,
 * called at src/integration/vanleer.pyx:32).  With is_prim=1 the primitives
 * are given and cons is derived on every cell (prim2cons); with is_prim=0
 * cons is given and prim is derived (cons2prim).  bfld may be NULL to keep
 * the current face field. */
int bnz_set_state(bnz_ctx* ctx, const double* prim_or_cons, int is_prim, const double* bfld);
/* init_sim after set_problem (src/integration/vanleer.pyx:41-48): ghost fill,
 * face-to-cell B, ghost fill of cell B, prim2cons everywhere; time = 0. */
int bnz_init(bnz_ctx* ctx);
/* Download (any pointer may be NULL): GridData.prim / cons / bfld. */
int bnz_get_state(bnz_ctx* ctx, double* prim, double* cons, double* bfld);

/* GridBC.apply_grid_bc(bvars) (src/bc/grid_bc.pyx:323-339): bit n of var_mask
 * selects prim variable n (0..8) or face component n-9 (9..11). */
int bnz_apply_bc(bnz_ctx* ctx, uint32_t var_mask);
/* BnzIntegr.new_dt (src/integration/new_dt.pyx:18-135): CFL time step. */
int bnz_new_dt(bnz_ctx* ctx, double* dt_out);
/* One VL2 step of size dt (src/integration/vanleer.pyx:101-163): predictor,
 * corrector, conduction (if kappa0 != 0), ghost fill, prim2cons. */
int bnz_vl2_step(bnz_ctx* ctx, double dt);
/* BnzDiffusion.diffuse (src/dissipation/diffusion.pyx:158-198): RKL2
 * super-time-stepped field-aligned conduction over dt.  *nsts_out (may be
 * NULL) receives the stage count. */
int bnz_diffuse(bnz_ctx* ctx, double dt, int* nsts_out);
/* vanleer.advance (src/integration/vanleer.pyx:59-179): step until time >=
 * tmax or max_steps (>0) steps.  The CFL step is computed and clipped to tmax
 * on the device; the host reads back 8 bytes per step to stop the loop. */
int bnz_advance(bnz_ctx* ctx, double tmax, int max_steps, double* time_out, long* step_out);
int bnz_get_time(bnz_ctx* ctx, double* time_out, long* step_out, double* last_dt);
/* RKL2 stages of the last conduction call (diffusion.pyx:217-224 get_nsts). */
int bnz_last_nsts(const bnz_ctx* ctx, int* nsts);
int bnz_set_time(bnz_ctx* ctx, double time, long step);
/* Sticky device error word (bits: 1 rho<=0, 2 p<=0, 4 NaN, 8 unordered
 * Riemann fan, 16 timeout); cleared by the call. */
int bnz_check(bnz_ctx* ctx, uint32_t* err_bits);
/* Wait for the context's stream. */
int bnz_sync(bnz_ctx* ctx);

/* vanleer.advance with the host out of the loop: one full step (CFL dt on the
 * device, clipped to tmax; FIXDT uses dt_fixed) is captured once into a CUDA
 * graph and replayed nsteps times without host synchronisation.  Steps after
 * time reaches tmax run with dt = 0.  Not available with conduction
 * (kappa0 > 0), whose stage count is chosen on the host. */
int bnz_advance_graph(bnz_ctx* ctx, double tmax, int nsteps);

/* Device pointers of the context's state (prim, cons, bfld), for zero-copy
 * interop; valid until bnz_destroy. */
int bnz_device_state(bnz_ctx* ctx, double** prim, double** cons, double** bfld);
/* Raw CUDA stream handle of the context (cudaStream_t as void*). */
int bnz_stream(bnz_ctx* ctx, void** stream);
/* Order the context's work on a caller-owned stream (cudaStream_t as void*;
 * NULL is the legacy default stream).  The caller keeps ownership. */
int bnz_set_stream(bnz_ctx* ctx, void* stream);
/* Number of kernels this context has launched so far. */
int bnz_launch_count(const bnz_ctx* ctx, long long* n);

/* ------------------------------------------------------------------------
 * Batches: many independent grids of uneven sizes (parameter sweeps) with
 * one shared method, advanced together -- each stage of a step is a single
 * launch over a tile list that spans every instance, each instance keeps its
 * own CFL time step, and steps are replayed from a CUDA graph.  No reference
 * counterpart: the reference runs one grid per process (vanleer.advance).
 * All 2D (the fused tile kernels; kappa0 = 0) or all 3D grids: the fused
 * chunk kernels over every instance in one launch per stage, or with
 * method->path = BNZ_PATH_SPLIT the split path's launches for each instance
 * in turn (faster per step on large grids); with kappa0 > 0 each instance's
 * RKL2 stages follow its own hyperbolic step over its own dt.
 * ------------------------------------------------------------------------ */
typedef struct bnz_batch bnz_batch;
int bnz_batch_create(const bnz_grid_desc* grids, int n, const bnz_method_desc* method, bnz_batch** out);
int bnz_batch_destroy(bnz_batch* batch);
const char* bnz_batch_last_error(const bnz_batch* batch);
int bnz_batch_size(const bnz_batch* batch, int* n);
/* The i-th instance as a context: bnz_set_state / bnz_init / bnz_get_state /
 * bnz_get_time / bnz_check work on it (do not step it on its own). */
int bnz_batch_instance(bnz_batch* batch, int i, bnz_ctx** ctx);
/* nsteps VL2 steps of every instance, each with its own CFL dt clipped to tmax. */
int bnz_batch_advance(bnz_batch* batch, double tmax, int nsteps);
/* The same steps launched one by one (no graph) with events around every
 * launch; ms_kernels[3] receives the mean duration in ms of the per-instance
 * dt launch, the predictor launch and the corrector launch.  For measurement. */
int bnz_batch_advance_timed(bnz_batch* batch, double tmax, int nsteps, double* ms_kernels);
/* Host-state stepping: loads every instance's state from host memory
 * (prim[q]: 9 fields, bfld[q]: 3 face fields, each over the instance's full
 * array with ghosts, as bnz_set_state takes them), advances nsteps steps with
 * per-instance CFL dt clipped to tmax, and writes the result back in place
 * with ghosts filled (as bnz_get_state(prim, NULL, bfld) returns it).  The
 * instances are split into nchunks groups of about equal size (0: 32) and
 * pipelined: the copy in of one group, the steps of the previous one and the
 * copy out of the one before that run at the same time on three streams.
 * Pinned host memory makes the copies asynchronous.  Returns when the copies
 * out are complete.  No counterpart in the reference, whose state lives in
 * host arrays between its steps (src/integration/vanleer.pyx:59-179). */
int bnz_batch_step_host(bnz_batch* batch, double* const* prim, double* const* bfld, double tmax, int nsteps,
                        int nchunks);
int bnz_batch_set_stream(bnz_batch* batch, void* stream);
/* Test switch, off unless a test turns it on; no counterpart in the
 * reference.  With on != 0 the persistent kernels (variants 6-9) arm their
 * TMA loads on the mbarriers but do not issue them, so every bounded wait for
 * staged input runs out (about a second each): the kernels flag the
 * instances' error words with the timeout bit (bnz_check then returns
 * BNZ_ERR_TIMEOUT) and leave without writing the tiles.  It makes a device
 * wait fail without a fault; the state it leaves is not a step's result. */
int bnz_batch_test_withhold_loads(bnz_batch* batch, int on);
int bnz_batch_launch_count(const bnz_batch* batch, long long* n);
int bnz_batch_sync(bnz_batch* batch);

/* Kernel variants (tile shape tx x ty, predictor staging, persistent
 * corrector fed by a tile queue with TMA-staged input) and the autotuner.
 * bnz_variant_count fills n and, if non-NULL, arrays of n entries.
 * bnz_batch_time_variant times `steps` steps of one variant on the live state
 * and restores the state afterwards; bnz_batch_autotune times every variant
 * and keeps the fastest (*best, and the per-variant ms, -1 where not built). */
int bnz_variant_count(int* n, int* tx, int* ty, int* staged, int* persistent);
int bnz_batch_set_variant(bnz_batch* batch, int variant);
int bnz_batch_get_variant(const bnz_batch* batch, int* variant);
int bnz_batch_time_variant(bnz_batch* batch, int variant, int steps, double* ms);
int bnz_batch_autotune(bnz_batch* batch, int steps, int* best, double* ms_per_variant);

/* ------------------------------------------------------------------------
 * Output support (src/io/output.pyx, src/io/io.pyx).
 * bnz_history fills out[16] with the reference's history row
 * (get_hst_vars_grid, output.pyx:20-140): step, time, <rho>, <E_kin>, <E_th>,
 * <E_mag>, <E>, <mx>, <my>, <mz>, <Bx>, <By>, <Bz>, rms(Bx), rms(By), rms(Bz)
 * (means over active cells), reduced on the device; it synchronises.
 * bnz_snapshot queues a copy of the current state (ghosts filled, cons derived)
 * into caller-owned host buffers of (9|9|3, Ntot) doubles (NULL skips one) and
 * returns at once: the copy drains on a separate stream while the next steps
 * run.  The host buffers must stay valid (page-locked for a true overlap)
 * until bnz_snapshot_wait returns. */
int bnz_history(bnz_ctx* ctx, double* out);
/* Divergence check of the face field, reduced on the device (synchronises):
 * out[0] = max over active cells of |div B| * dx, with div B the sum over
 * the cell's faces of (b_upper - b_lower) / face spacing; out[1] = max |B| of
 * the cell-centred field.  out[0] / out[1] is the relative divergence that
 * constrained transport keeps at round-off (the face update of
 * src/integration/ct.pyx:15-91).  The reference computes it only in
 * commented-out checks (src/problem/weakshock.pyx:202-205). */
int bnz_div_b(bnz_ctx* ctx, double* out);
int bnz_snapshot(bnz_ctx* ctx, double* prim, double* cons, double* bfld);
int bnz_snapshot_wait(bnz_ctx* ctx);

/* ------------------------------------------------------------------------
 * Discrete adjoint of the VL2 step (fused 2D path, PLM with or without
 * charact_proj, rsolver hll, hllt or hlld, constant gravity; no conduction or
 * turbulence driving; fixed dt).  No counterpart in the reference, which has no
 * adjoint; these serve the torch.autograd wrapper (bonzo_b200/adjoint.py).
 * All state and cotangent pointers are DEVICE pointers to full arrays with
 * ghosts, (9, Ntot) prim and (3, Ntot) face field, ordered on the context's
 * stream.  A cotangent of an output refers to the arrays as
 * bnz_get_state_device returns them (ghosts filled); the cotangent of an input
 * is zero on ghost entries, which the step never reads. */

/* Device-to-device state copies (bnz_set_state / bnz_get_state with device
 * buffers; set takes prim and derives cons). */
int bnz_set_state_device(bnz_ctx* ctx, const double* prim, const double* bfld);
int bnz_get_state_device(bnz_ctx* ctx, double* prim, double* bfld);
/* nsteps steps of fixed dt from the current state, keeping the input state of
 * every checkpoint_every-th step on the device (the tape for the reverse pass). */
int bnz_rollout_forward(bnz_ctx* ctx, int nsteps, double dt, int checkpoint_every);
/* Reverse pass of the recorded rollout: cotangent of the final state ->
 * cotangent of the initial state.  Segments between checkpoints are recomputed;
 * the context's state is left at the rollout's final state. */
int bnz_rollout_adjoint(bnz_ctx* ctx, const double* gprim, const double* gbfld, double* gprim0, double* gbfld0);
/* VJP of one step of dt at the state (prim, bfld): cotangent of the step's
 * output (gprim1, gbfld1) -> cotangent of its input (gprim0, gbfld0).  The
 * context's state becomes the step's output. */
int bnz_step_adjoint(bnz_ctx* ctx, double dt, const double* prim, const double* bfld, const double* gprim1,
                     const double* gbfld1, double* gprim0, double* gbfld0);

/* ------------------------------------------------------------------------
 * One VL2 step that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that must not let a library allocate --
 * programs whose device memory belongs to a framework allocator that reserved
 * it up front, or time loops that cannot take the device-wide synchronisation
 * of a cudaMalloc / cudaFree.  The caller passes device pointers to full
 * (ghosts included) prim / bfld arrays: the input state and the output state.
 * The outputs must not overlap the inputs or each other (BNZ_ERR_ARG).  The
 * step (predictor + corrector + ghost fill of the outputs, no conduction)
 * keeps its scratch in one fixed 4 MiB device array that every GPU loading the
 * library holds until exit, which bounds the grid to 2D with (Nx+6)*(Ny+6) up
 * to about 40000 cells (e.g. 192 x 192, PLM); larger grids are rejected with
 * BNZ_ERR_ARG.  lmax[2] - lmin[2] is the depth of the single z cell and must
 * be positive.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * A call queues its kernels on `stream` (cudaStream_t as void*, NULL for the
 * legacy stream) and returns without waiting for the GPU; the descriptor, tile
 * list and coordinates are written into the array by a set-up kernel.  All
 * calls share the array: calls that overlap on the GPU race and corrupt each
 * other.  The message of the last failure on this host thread is
 * bnz_noalloc_last_error(). */
int bnz_vl2_step_noalloc(const bnz_grid_desc* grid, const bnz_method_desc* method, const double* prim_in,
                         const double* bfld_in, double* prim_out, double* bfld_out, double dt, void* stream);
const char* bnz_noalloc_last_error(void);
/* Error word of the no-alloc steps queued so far (bits as bnz_check: 1 rho<=0,
 * 2 p<=0, 4 NaN, 8 unordered Riemann fan, 16 timeout): sticky across steps,
 * read and cleared by this call, which waits for `stream`.  Returns BNZ_OK,
 * BNZ_ERR_STATE or BNZ_ERR_TIMEOUT as bnz_check does.  No counterpart in the
 * reference. */
int bnz_noalloc_check(void* stream, uint32_t* err_bits);
/* Size in bytes of the fixed scratch array. */
size_t bnz_noalloc_scratch_bytes(void);

/* The reference's C-level Riemann call (src/mhd/fluxes_c.h:3-20: hll_flux,
 * hllc_flux, hllt_flux, hlld_flux(flux, wL, wR, bx, i1, i2, gam) over row
 * pointers) on DEVICE rows: n interfaces, row q of wl / wr / flux at
 * [q * n .. q * n + n), bx[n] the face-normal field.  nvar = 9 for MHD builds
 * (wL[BX] = wR[BX] = bx) or 6 for the hydro build (rho, v, p, passive scalar;
 * bx unused, hll takes the hydro sound speed, hllc available).  exact_fp
 * selects the kernels built without multiply-add contraction.  Queued on
 * `stream`; *err_bits (a device word, may be NULL) receives the fan-ordering
 * flags OR-ed in. */
int bnz_riemann(int rsolver, int nvar, const double* wl, const double* wr, const double* bx, double* flux, int n,
                double gam, int exact_fp, unsigned* err_bits, void* stream);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (fma chains
 * on every SM), the denominator of the kernels' FP64-pipe fraction.  No
 * counterpart in the reference: a measurement helper. */
int bnz_fp64_fma_peak(double* tflops);

/* y[q] = 1 / x[q] (device arrays of n doubles, queued on `stream`) by the
 * reciprocal the fast build uses in place of a division (the van Leer
 * limiter's): an approximate hardware reciprocal refined by two Newton-Raphson
 * steps.  For normal x it is within 2 ulp of the IEEE quotient; the tests
 * check that bound.  No counterpart in the reference: a check helper. */
int bnz_fast_rcp(const double* x, double* y, int n, void* stream);

#ifdef __cplusplus
}
#endif

#endif
