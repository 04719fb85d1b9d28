// bnz_noalloc.cu -- one VL2 step that allocates no device memory.
//
// For callers that must not allocate device memory while they run: programs
// whose device memory is handed out by a framework allocator that reserved it
// up front (so a library's own cudaMalloc fails or fragments the pool), and
// time loops that cannot afford the device-wide synchronisation a cudaMalloc /
// cudaFree implies.  Such a caller owns every input and output buffer; the
// step's own working memory lives in one file-scope device array of a fixed
// size that every GPU loading this library holds until the process exits.
//
// The step is the fused 2D predictor + corrector of the batch path run on one
// grid; its scratch (predictor state, time record, error word, coordinates,
// grid descriptor and tile list) is carved out of that array.  A call queues
// work and returns: a set-up kernel that takes its parameters by value writes
// the descriptor, time record, tiles and coordinates into the array, so no
// host buffer is copied and the host never waits.  All calls share the array:
// two calls whose work overlaps on the GPU (different streams, or different
// host threads) race on it and corrupt each other's results.  The error word
// is sticky across calls until bnz_noalloc_check reads and clears it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bnz_gpu.h"
#include "bnz_common.h"
#include "bnz_launch.h"

namespace {

// 4 MiB of scratch: enough for grids with (Nx+6)*(Ny+6) up to about 40000
// cells, e.g. 192 x 192 active cells with the three ghost layers of PLM.
constexpr size_t kScratchBytes = 4u << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_mu;
thread_local std::string g_err;

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

int fail(int code, const std::string& m) {
  g_err = m;
  return code;
}

// Device address of g_scratch on the current device.  In host code the name
// g_scratch is only a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress, once per device, on the first call made with that
// device current.
int scratch_address(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(BNZ_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(BNZ_ERR_UNSUPPORTED, "device index above 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return fail(BNZ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[dev];
  return BNZ_OK;
}

// Everything a call needs in the scratch array besides the predictor state,
// passed by value to one set-up kernel: no host buffer is read after the call
// returns, so nothing is uploaded and nothing waits for the GPU.
struct Setup {
  FusedInst inst;      // its pointers already refer to the scratch array
  FusedInst* d_inst;   // where the descriptor goes
  DtState* d_ds;       // the time record: dt of this step, no tmax clip
  double dt;
  FusedTile* d_tiles;  // predictor tiles, then corrector tiles
  int ntA, ntB;
  int N[2], ng, tx, ty;
  double* coord[3];    // 5 arrays of Ntot + 1 per axis: dlf, dlf_inv, lf, lv, dlv_inv
  int Ntot[3], ind1[3], ind2[3];
  double lmin[3], lmax[3];
  int bc[3][2];
};

// Tile t of one list (variant 0 tiles; the predictor's cover cells
// 1..Ntot-2, the corrector's the active cells), as make_tiles builds them.
__device__ FusedTile tile_of(const Setup& p, int t, bool pred) {
  const int T[2] = {p.tx, p.ty};
  int nt[2];
  for (int a = 0; a < 2; ++a) nt[a] = (p.N[a] + T[a] - 1) / T[a];
  const int b[2] = {t % nt[0], t / nt[0]};
  int lo[2], hi[2];
  for (int a = 0; a < 2; ++a) {
    lo[a] = p.ng + b[a] * T[a];
    hi[a] = min(p.ng + (b[a] + 1) * T[a], p.ng + p.N[a]) - 1;
    if (pred) {
      if (b[a] == 0) lo[a] = 1;
      if (b[a] == nt[a] - 1) hi[a] = p.N[a] + 2 * p.ng - 2;
    }
  }
  FusedTile r;
  r.inst = 0;
  r.x0 = lo[0];
  r.y0 = lo[1];
  r.wx = hi[0] - lo[0] + 1;
  r.wy = hi[1] - lo[1] + 1;
  r.tma = 0;
  return r;
}

// One block.  The coordinates follow coord.pyx:122-258 and cartesian.pyx:18-43
// with the context's host arithmetic operation for operation (explicitly
// rounded adds, multiplies and divisions, never contracted), so the step is
// bitwise the context's.  The error word is left alone: it is sticky until
// bnz_noalloc_check reads it.
__global__ void k_noalloc_setup(Setup p) {
  if (threadIdx.x == 0) {
    *p.d_inst = p.inst;
    DtState ds;
    memset(&ds, 0, sizeof ds);
    ds.dt = p.dt;
    ds.tmax = 1e300;
    *p.d_ds = ds;
  }
  for (int t = threadIdx.x; t < p.ntA + p.ntB; t += blockDim.x)
    p.d_tiles[t] = t < p.ntA ? tile_of(p, t, true) : tile_of(p, t - p.ntA, false);
  // face coordinates: the uniform formula, then the ghost spacings of
  // periodic / reflecting boundaries (sequential: each face uses the next one)
  for (int a = 0; a < 3; ++a) {
    const int len = p.Ntot[a] + 1;
    double* lf = p.coord[a] + 2 * (size_t)len;
    if (p.Ntot[a] == 1) {
      if (threadIdx.x == 0) {
        lf[0] = p.lmin[a];
        lf[1] = p.lmax[a];
      }
      continue;
    }
    const int nact = p.ind2[a] - p.ind1[a] + 1;
    const double dx = __ddiv_rn(__dsub_rn(p.lmax[a], p.lmin[a]), (double)nact);
    const double l1 = __dmul_rn(__dmul_rn(0., (double)nact), dx);
    for (int i = threadIdx.x; i < len; i += blockDim.x) lf[i] = __dadd_rn(l1, __dmul_rn((double)(i - p.ind1[a]), dx));
  }
  __syncthreads();
  if (threadIdx.x < 3 && p.Ntot[threadIdx.x] > 1) {
    const int a = threadIdx.x, Ntot = p.Ntot[a], i1 = p.ind1[a], i2 = p.ind2[a];
    double* lf = p.coord[a] + 2 * (size_t)(Ntot + 1);
    if (p.bc[a][0] == BNZ_BC_PERIODIC)
      for (int i = i1 - 1; i > -1; --i) {
        const int j = i2 - i + (i1 - 1);
        lf[i] = __dsub_rn(lf[i + 1], __dsub_rn(lf[j + 1], lf[j]));
      }
    if (p.bc[a][1] == BNZ_BC_PERIODIC)
      for (int i = i2 + 1; i < Ntot; ++i) {
        const int j = i1 + i - (i2 + 1);
        lf[i + 1] = __dadd_rn(lf[i], __dsub_rn(lf[j + 1], lf[j]));
      }
    if (p.bc[a][0] == BNZ_BC_REFLECT)
      for (int i = i1 - 1; i > -1; --i) {
        const int j = i1 - i + (i1 - 1);
        lf[i] = __dsub_rn(lf[i + 1], __dsub_rn(lf[j + 1], lf[j]));
      }
    if (p.bc[a][1] == BNZ_BC_REFLECT)
      for (int i = i2 + 1; i < Ntot; ++i) {
        const int j = i2 - i + (i2 + 1);
        lf[i + 1] = __dadd_rn(lf[i], __dsub_rn(lf[j + 1], lf[j]));
      }
  }
  __syncthreads();
  // spacings and centres (the last entry of each array stays 0, dlv_inv[0] too)
  for (int a = 0; a < 3; ++a) {
    const int Ntot = p.Ntot[a], len = Ntot + 1;
    double* dlf = p.coord[a];
    double* dlfi = dlf + len;
    const double* lf = dlf + 2 * (size_t)len;
    double* lv = dlf + 3 * (size_t)len;
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
      if (i < Ntot) {
        const double d = __dsub_rn(lf[i + 1], lf[i]);
        dlf[i] = d;
        dlfi[i] = __ddiv_rn(1., d);
        lv[i] = __dmul_rn(0.5, __dadd_rn(lf[i], lf[i + 1]));
      } else {
        dlf[i] = dlfi[i] = lv[i] = 0.;
      }
    }
  }
  __syncthreads();
  for (int a = 0; a < 3; ++a) {
    const int Ntot = p.Ntot[a], len = Ntot + 1;
    const double* lv = p.coord[a] + 3 * (size_t)len;
    double* dlvi = p.coord[a] + 4 * (size_t)len;
    for (int i = threadIdx.x; i < len; i += blockDim.x)
      dlvi[i] = (i >= 1 && i < Ntot) ? __ddiv_rn(1., __dsub_rn(lv[i], lv[i - 1])) : 0.;
  }
}

// Tile counts of variant 0 (the predictor's list, then the corrector's).
int tiles_count(int N, int t) { return (N + t - 1) / t; }

bool overlap(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + nb && y < x + na;
}

}  // namespace

extern "C" {

int bnz_vl2_step_noalloc(const bnz_grid_desc* g, const bnz_method_desc* m, const double* prim_in,
                         const double* bfld_in, double* prim_out, double* bfld_out, double dt, void* stream) {
  if (!g || !m || !prim_in || !bfld_in || !prim_out || !bfld_out) return fail(BNZ_ERR_ARG, "null argument");
  if (g->dims != 2 || g->Nz != 1) return fail(BNZ_ERR_UNSUPPORTED, "the no-alloc step covers 2D grids");
  if (m->reconstr != BNZ_RCN_LINEAR) return fail(BNZ_ERR_UNSUPPORTED, "the no-alloc step uses PLM (reconstr linear)");
  if (m->kappa0 != 0.) return fail(BNZ_ERR_UNSUPPORTED, "the no-alloc step has no conduction (kappa0 = 0)");
  if (m->drive_f0 != 0.) return fail(BNZ_ERR_UNSUPPORTED, "the no-alloc step has no turbulence driving (drive_f0 = 0)");
  if (m->rsolver != BNZ_RS_HLL && m->rsolver != BNZ_RS_HLLD && m->rsolver != BNZ_RS_HLLT)
    return fail(BNZ_ERR_ARG, "rsolver must be hll, hlld or hllt");
  if (m->limiter < 0 || m->limiter > 2) return fail(BNZ_ERR_ARG, "limiter must be vl, mc or mm");
  if (!(m->gam > 1.)) return fail(BNZ_ERR_ARG, "gam must exceed 1");
  if (!(dt > 0.) || std::isinf(dt)) return fail(BNZ_ERR_ARG, "dt must be finite and > 0");
  const int ng = 3;
  if (g->Nx < ng || g->Ny < ng) return fail(BNZ_ERR_ARG, "each axis needs at least 3 active cells");
  for (int a = 0; a < 3; ++a) {
    // the z extent is the depth of the single z cell (face areas and volumes)
    if (!(g->lmax[a] > g->lmin[a])) return fail(BNZ_ERR_ARG, "lmax must exceed lmin on every axis (z: the cell depth)");
    for (int sd = 0; sd < 2; ++sd)
      if (g->bc[a][sd] < 0 || g->bc[a][sd] > 2) return fail(BNZ_ERR_ARG, "bc flag must be 0, 1 or 2");
    if (a < 2 && (g->bc[a][0] == BNZ_BC_PERIODIC) != (g->bc[a][1] == BNZ_BC_PERIODIC))
      return fail(BNZ_ERR_ARG, "periodic boundaries must be set on both sides of an axis");
  }
  const int nx = g->Nx + 2 * ng, ny = g->Ny + 2 * ng;
  const size_t ncell = (size_t)nx * ny;
  const FusedVariant& v = FUSED_VARIANTS[0];
  const int ntA = tiles_count(g->Nx, v.tx) * tiles_count(g->Ny, v.ty);
  const int ntB = ntA;
  // layout of the scratch array
  const size_t o_inst = 0;
  const size_t o_ds = align256(o_inst + sizeof(FusedInst));
  const size_t o_err = align256(o_ds + sizeof(DtState));
  const size_t o_tiles = align256(o_err + sizeof(unsigned));
  const size_t o_coord = align256(o_tiles + (size_t)(ntA + ntB) * sizeof(FusedTile));
  const size_t ncoord = 5 * (size_t)(nx + 1) + 5 * (size_t)(ny + 1) + 5 * 2;
  const size_t o_ws = align256(o_coord + ncoord * sizeof(double));
  const size_t o_bs = align256(o_ws + 9 * ncell * sizeof(double));
  const size_t need = align256(o_bs + 3 * ncell * sizeof(double));
  if (need > kScratchBytes)
    return fail(BNZ_ERR_ARG, "grid too large for the no-alloc step: it needs " + std::to_string(need) +
                                 " bytes of scratch and the fixed array holds " + std::to_string(kScratchBytes) +
                                 " ((Nx+6)*(Ny+6) must stay below about 40000 cells)");
  // inputs are read while outputs are written: no output may share memory
  // with an input or with the other output
  const size_t pb = 9 * ncell * sizeof(double), bb = 3 * ncell * sizeof(double);
  if (overlap(prim_in, pb, prim_out, pb) || overlap(prim_in, pb, bfld_out, bb) ||
      overlap(bfld_in, bb, prim_out, pb) || overlap(bfld_in, bb, bfld_out, bb) || overlap(prim_out, pb, bfld_out, bb))
    return fail(BNZ_ERR_ARG, "output buffers must not overlap the input buffers or each other");
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;

  Setup p;
  memset(&p, 0, sizeof p);
  // coordinates (x, y, and the single z cell), 5 arrays of Ntot + 1 per axis
  double* dcoord = reinterpret_cast<double*>(base + o_coord);
  const double* ptr[3][5];
  {
    size_t off = 0;
    const int N[3] = {nx, ny, 1};
    const int i1[3] = {ng, ng, 0}, i2[3] = {ng + g->Nx - 1, ng + g->Ny - 1, 0};
    for (int a = 0; a < 3; ++a) {
      const size_t len = (size_t)N[a] + 1;
      p.coord[a] = dcoord + off;
      p.Ntot[a] = N[a];
      p.ind1[a] = i1[a];
      p.ind2[a] = i2[a];
      p.lmin[a] = g->lmin[a];
      p.lmax[a] = g->lmax[a];
      p.bc[a][0] = g->bc[a][0];
      p.bc[a][1] = g->bc[a][1];
      for (int q = 0; q < 5; ++q) ptr[a][q] = dcoord + off + q * len;
      off += 5 * len;
    }
  }
  FusedInst& I = p.inst;
  I.nx = nx;
  I.ny = ny;
  I.N[0] = g->Nx;
  I.N[1] = g->Ny;
  I.ng = ng;
  I.sv = (long long)ncell;
  I.gam = m->gam;
  for (int a = 0; a < 2; ++a) {
    I.bc[a][0] = g->bc[a][0];
    I.bc[a][1] = g->bc[a][1];
    I.dlf[a] = ptr[a][0];
    I.dlf_inv[a] = ptr[a][1];
    I.lf[a] = ptr[a][2];
    I.lv[a] = ptr[a][3];
  }
  I.face_aware = m->outflow_face_aware;
  I.dlf2 = g->lmax[2] - g->lmin[2];  // the single z cell of a 2D grid
  I.w[0] = const_cast<double*>(prim_in);
  I.w[1] = prim_out;
  I.b[0] = const_cast<double*>(bfld_in);
  I.b[1] = bfld_out;
  I.ws = reinterpret_cast<double*>(base + o_ws);
  I.bs = reinterpret_cast<double*>(base + o_bs);
  I.ds = reinterpret_cast<DtState*>(base + o_ds);
  I.err = reinterpret_cast<unsigned*>(base + o_err);
  for (int d = 0; d < 3; ++d) I.grav[d] = m->grav[d];
  I.src = (m->grav[0] != 0. || m->grav[1] != 0. || m->grav[2] != 0.) ? 1 : 0;
  p.d_inst = reinterpret_cast<FusedInst*>(base + o_inst);
  p.d_ds = I.ds;
  p.dt = dt;
  p.d_tiles = reinterpret_cast<FusedTile*>(base + o_tiles);
  p.ntA = ntA;
  p.ntB = ntB;
  p.N[0] = g->Nx;
  p.N[1] = g->Ny;
  p.ng = ng;
  p.tx = v.tx;
  p.ty = v.ty;
  k_noalloc_setup<<<1, 256, 0, s>>>(p);

  const Launchers* L = m->exact_fp ? &exact::table : &fast::table;
  FusedLaunch f;
  memset(&f, 0, sizeof f);
  f.insts = p.d_inst;
  f.ninst = 1;
  f.tilesA = p.d_tiles;
  f.ntA = ntA;
  f.tilesB = f.tilesA + ntA;
  f.ntB = ntB;
  f.rsolver = m->rsolver;
  f.limiter = m->limiter;
  f.charact_proj = m->charact_proj;
  f.variant = 0;
  f.cour = m->cour;
  f.dt_mode = FDT_EXPLICIT;
  f.stream = s;
  L->fused_step(f, 0);
  // ghost fill of the outputs (vanleer.pyx:162) so they are complete arrays
  StepArgs a;
  memset(&a, 0, sizeof a);
  GridDev& gd = a.g;
  gd.nx = nx;
  gd.ny = ny;
  gd.nz = 1;
  gd.dims = 2;
  gd.ng = ng;
  gd.i1 = ng;
  gd.i2 = ng + g->Nx - 1;
  gd.j1 = ng;
  gd.j2 = ng + g->Ny - 1;
  gd.k1 = gd.k2 = 0;
  gd.sv = (long long)ncell;
  gd.gam = m->gam;
  for (int ax = 0; ax < 3; ++ax) {
    gd.dlf[ax] = ptr[ax][0];
    gd.dlf_inv[ax] = ptr[ax][1];
    gd.lf[ax] = ptr[ax][2];
    gd.lv[ax] = ptr[ax][3];
    gd.dlv_inv[ax] = ptr[ax][4];
  }
  for (int x = 0; x < 3; ++x) {
    a.bc[x][0] = g->bc[x][0];
    a.bc[x][1] = g->bc[x][1];
  }
  a.face_aware = m->outflow_face_aware;
  a.stream = s;
  L->apply_bc(a, prim_out, bfld_out, 0xFFFu);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BNZ_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return BNZ_OK;
}

int bnz_noalloc_check(void* stream, uint32_t* err_bits) {
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // the error word sits at the same place for every grid (after the
  // descriptor and the time record)
  unsigned* d_err = reinterpret_cast<unsigned*>(base + align256(align256(sizeof(FusedInst)) + sizeof(DtState)));
  unsigned h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, d_err, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(BNZ_ERR_CUDA, std::string("error word: ") + cudaGetErrorString(e));
  if (err_bits) *err_bits = h;
  if (h & 16u) return fail(BNZ_ERR_TIMEOUT, "a bounded device wait ran out");
  if (h) return fail(BNZ_ERR_STATE, "non-physical state on the device (error bits " + std::to_string(h) + ")");
  return BNZ_OK;
}

const char* bnz_noalloc_last_error(void) { return g_err.c_str(); }

size_t bnz_noalloc_scratch_bytes(void) { return kScratchBytes; }

}  // extern "C"
