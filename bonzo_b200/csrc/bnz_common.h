// bnz_common.h -- structures shared by the host context and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Grid geometry as the kernels see it.  Index conventions follow the
// reference's GridCoord (src/coordinates/coord_c.h:19-99): Ntot cells per axis
// including ng ghosts on active axes, active range i1..i2 / j1..j2 / k1..k2,
// per-axis spacing arrays indexed by the cell index along that axis.
struct GridDev {
  int nx, ny, nz;     // Ntot per axis
  int dims, ng;
  int i1, i2, j1, j2, k1, k2;
  long long sv;       // stride between variables: nx*ny*nz
  double gam;
  const double* dlf[3];      // face spacing lf[i+1]-lf[i]
  const double* dlf_inv[3];
  const double* lf[3];       // face coordinates (Ntot+1 entries)
  const double* lv[3];       // volume (centre) coordinates
  const double* dlv_inv[3];  // inverse centre spacing
};

// Device buffers and options used by one step of one grid.
struct StepArgs {
  GridDev g;
  double* prim;
  double* cons;
  double* bfld;
  double* cons_s;  // predictor conserved state (plain path)
  double* bfld_s;  // predictor face field (plain path)
  double* flx[3];  // Godunov fluxes (plain path)
  double* ec;      // cell-centred E (plain path)
  double* ee;      // edge E (plain path)
  double* wnext;   // fused path: output prim buffer
  double* bnext;   // fused path: output face-B buffer
  unsigned* err;   // sticky device error word
  int rsolver, reconstr_order, limiter, charact_proj;
  int bc[3][2];
  int face_aware;
  cudaStream_t stream;
  // source terms: constant gravity and the driving force field (3 x Ntot)
  double grav[3];
  const double* fdriv;
  int src;  // any source term on
  int hydro;  // the reference's hydro build (MFIELD 0): no field, no CT
  // split path, 3D grids with even Ntot_x: the tensor maps of the update
  // kernel's TMA boxes (split::TM_COUNT maps of 128 bytes), or null
  const unsigned char* smaps;
};

// Device time-step record used by graph-captured stepping.
struct DtState {
  double dt;          // step used by the current step
  double time;        // simulation time after the last completed step
  double tmax;        // clip target
  unsigned long long cdsmax_bits;  // max of (|v|+cf)/dx as a bit pattern
  long long step;
  unsigned long long cds_bits[2];  // fused path: CFL max of the state of parity p
};

// Fused 2D path: one grid ("instance") of a batch, as the kernels see it.
struct FusedInst {
  int nx, ny;          // Ntot (x, y)
  int N[2];            // active cells
  int ng;
  long long sv;        // variable stride nx*ny
  double gam;
  int bc[2][2];
  int face_aware;
  const double* dlf[2];
  const double* dlf_inv[2];
  const double* lf[2];
  const double* lv[2];
  double dlf2;         // z extent of the single z cell
  double* w[2];        // prim, ping-pong by step parity
  double* b[2];        // face field, ping-pong
  double* ws;          // predictor prim
  double* bs;          // predictor face field
  DtState* ds;
  unsigned* err;       // the instance's sticky error word
  double grav[3];      // source terms (gravity, driving force field or null)
  const double* fdriv;
  int src;
};

// Fused 3D path: one grid of a 3D batch (or a single 3D context).
struct FusedInst3 {
  int nx, ny, nz;      // Ntot per axis
  int N[3];            // active cells
  int ng;
  long long sv;        // variable stride nx*ny*nz
  double gam;
  int bc[3][2];
  int face_aware;
  const double* dlf[3];
  const double* dlf_inv[3];
  const double* lf[3];
  const double* lv[3];
  double* w[2];        // prim, ping-pong by step parity
  double* b[2];        // face field, ping-pong
  double* ws;          // predictor prim
  double* bs;          // predictor face field
  DtState* ds;
  unsigned* err;
  double grav[3];
  const double* fdriv;
  int src;
};

// Chunk shape of the 3D kernels: at most F3_TX x F3_TY cells in x, y and about
// F3_KZ planes (16 x 8 on one 512-thread block per SM: the flux phase of a
// plane is one round, and the halo recompute of x and y faces stays at one
// Riemann solve per cell and direction plus a third); the corrector's TMA box
// of ws covers the chunk plus two cells each side from an even column:
// F3_BW x F3_BH cells, one plane, 9 fields.
constexpr int F3_TX = 16, F3_TY = 8, F3_KZ = 64;
constexpr int F3_BW = (F3_TX + 6) & ~1, F3_BH = F3_TY + 4;

// A column chunk of a 3D grid: cells [x0, x0+wx) x [y0, y0+wy) x [z0, z0+wz).
struct FusedTile3 {
  int inst;
  int x0, y0, z0;
  int wx, wy, wz;
  int tma;  // the corrector stages ws by TMA (the instance has a tensor map)
};

struct Fused3Launch {
  const FusedInst3* insts;
  int ninst;
  const FusedTile3* tilesA;  // predictor chunks (cells 1..Ntot-2 of each axis)
  int ntA;
  const FusedTile3* tilesB;  // corrector chunks (active cells)
  int ntB;
  int rsolver, limiter, charact_proj;
  double cour;
  int dt_mode;
  double dt_fixed;
  const unsigned char* wsmaps;  // per-instance 4D tensor maps of ws (128 bytes each), or null
  cudaStream_t stream;
  cudaEvent_t* events;  // optional: before dt, predictor, corrector and after (timing)
};

// A tile of cells [x0, x0+wx) x [y0, y0+wy) (array coordinates) of one instance.
struct FusedTile {
  int inst;
  int x0, y0;
  int wx, wy;
  int tma;  // the instance has a tensor map of its ws (persistent corrector)
};

// Variants of the fused kernels the autotuner chooses from: tile shape
// (cells along x, y), whether the predictor stages its input cells in shared
// memory, and whether the stages run as persistent TMA-fed kernels.  A batch
// starts on variant 8 (persistent, 15 x 14), a single grid on variant 0
// (32 x 8: fewer tiles, one wave on a 256^2 grid).
struct FusedVariant {
  int tx, ty, staged, persistent;
};
// 15 x 14 tiles give 256 x faces and 255 y faces per interior tile: each flux
// phase of a 256-thread block is one full round (32 x 8 leaves 40% of the
// threads idle in the second round of each phase).
// The persistent variants run the corrector (persistent = 1) or both stages
// (2) as one resident grid fed by a tile queue, with TMA double-buffering of
// the staged input (15 x 14 only: two blocks of those kernels fit one SM's
// shared memory).
// 14 x 14 tiles (variant 9) make every phase of the corrector at most one
// round: 256 slope cells, 240 x and 240 y faces, 225 corners, 196 cells.
constexpr int FUSED_NVARIANT = 10;
constexpr FusedVariant FUSED_VARIANTS[FUSED_NVARIANT] = {
    {32, 8, 0, 0}, {32, 8, 1, 0}, {16, 16, 0, 0}, {16, 16, 1, 0}, {15, 14, 0, 0},
    {15, 14, 1, 0}, {15, 14, 0, 1}, {15, 14, 1, 1}, {15, 14, 0, 2}, {14, 14, 0, 2}};

// Variants built for a Riemann solver: all for HLLD; the default and the
// persistent variants 8 and 9 for the others.
inline bool fused_variant_built(int v, bool hlld) {
  return v == 0 || v == 8 || v == 9 || (hlld && v > 0 && v < FUSED_NVARIANT);
}

constexpr int BATCH_DEFAULT_VARIANT = 8;

// dt modes of the fused step
enum { FDT_CFL = 0, FDT_EXPLICIT = 1, FDT_FIXED = 2 };

struct FusedLaunch {
  const FusedInst* insts;   // indexed by the tiles' instance numbers
  int ninst;                // the per-instance launches cover insts[inst0 .. inst0+ninst-1]
  int inst0;
  const FusedTile* tilesA;  // predictor tiles (cells 1..Ntot-2 of each axis)
  int ntA;
  const FusedTile* tilesB;  // corrector tiles (active cells)
  int ntB;
  int rsolver, limiter, charact_proj;
  int variant;
  double cour;
  int dt_mode;
  double dt_fixed;
  unsigned* err;
  cudaStream_t stream;
  // persistent kernels: per-instance tensor maps (128 bytes each) of ws
  // (corrector) and of w[0], w[1] (predictor), and the two work-queue
  // counters (corrector, predictor); null where the variant does not use them
  const unsigned char* wsmaps;
  const unsigned char* wmaps;
  unsigned* queue;
  int withhold;  // test switch: the persistent kernels' TMA loads are not issued
  // optional: events recorded before k_dt_batch, before the predictor, before
  // the corrector and after it (kernel timing; null in normal stepping)
  cudaEvent_t* events;
};

// One reverse (adjoint) step of the fused 2D path: the recorded forward
// values, the incoming and outgoing cotangents and the scratch.
struct AdjStep {
  const double* Wn;   // w^n, b^n (the step's input state)
  const double* Bn;
  const double* Ws;   // ws, bs (the predictor's output for that state)
  const double* Bs;
  const double* W1;   // w^(n+1) (the step's output prim)
  double* G1w;        // cotangent of the output (folded in place first)
  double* G1b;
  double* Vw;         // out: cotangent of the input state (9 + 3 fields)
  double* Vb;
  double* Wsb;        // scratch: 9, 3, 9, 1 and 72 fields of Ntot cells
  double* Bsb;
  double* Ub;
  double* Eb;
  double* Q;
  double dt;
  int rsolver, limiter;
  int charact;        // the corrector's slopes are projected (charact_proj)
  int fold_in;        // fold G1 first (it may carry ghost entries)
  int clear_bsb;      // zero Bsb first (the first reverse step of a pass)
  cudaStream_t stream;
};

// Turbulence driving (turb_driv.pyx): force field, this step's mode
// amplitudes (device), base wavenumbers 2 pi / L and the OU parameters.
struct DriveArgs {
  double* fdriv;
  const double* modes;
  int nmod;
  double k0[3];
  double tau, f0;
};

// Conduction scratch (thcond_elec.pyx DiffScratch).
struct DiffArgs {
  double* temp;
  double* fx;
  double* fy;
  double* fz;
  double* pres0;
  double* presm1;
  double* dtemp;
  double* dtemp0;
  double kappa0;
  int aniso, sat;
  double cour_diff;
};
