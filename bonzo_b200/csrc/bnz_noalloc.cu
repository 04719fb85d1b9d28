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
// grid descriptor and tile list) is carved out of that array.  All calls share
// the array: two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it and corrupt each other's results.
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

// Face coordinates and spacings of one axis (coord.pyx:122-258,
// cartesian.pyx:18-43); every array has Ntot+1 entries.
void axis_coords(int n, int Ntot, int ind1, int ind2, const bnz_grid_desc* g, std::vector<double>& lf,
                 std::vector<double>& lv, std::vector<double>& dlf, std::vector<double>& dlfi,
                 std::vector<double>& dlvi) {
  lf.assign(Ntot + 1, 0.);
  if (Ntot == 1) {
    lf[0] = g->lmin[n];
    lf[1] = g->lmax[n];
  } else {
    int Nact = ind2 - ind1 + 1;
    double dx = (g->lmax[n] - g->lmin[n]) / Nact;
    double l1 = 0 * Nact * dx;
    for (int i = 0; i < Ntot + 1; ++i) lf[i] = l1 + (i - ind1) * dx;
    if (g->bc[n][0] == BNZ_BC_PERIODIC)
      for (int i = ind1 - 1; i > -1; --i) {
        int i_ = ind2 - i + (ind1 - 1);
        double d = lf[i_ + 1] - lf[i_];
        lf[i] = lf[i + 1] - d;
      }
    if (g->bc[n][1] == BNZ_BC_PERIODIC)
      for (int i = ind2 + 1; i < Ntot; ++i) {
        int i_ = ind1 + i - (ind2 + 1);
        double d = lf[i_ + 1] - lf[i_];
        lf[i + 1] = lf[i] + d;
      }
    if (g->bc[n][0] == BNZ_BC_REFLECT)
      for (int i = ind1 - 1; i > -1; --i) {
        int i_ = ind1 - i + (ind1 - 1);
        double d = lf[i_ + 1] - lf[i_];
        lf[i] = lf[i + 1] - d;
      }
    if (g->bc[n][1] == BNZ_BC_REFLECT)
      for (int i = ind2 + 1; i < Ntot; ++i) {
        int i_ = ind2 - i + (ind2 + 1);
        double d = lf[i_ + 1] - lf[i_];
        lf[i + 1] = lf[i] + d;
      }
  }
  lv.assign(Ntot + 1, 0.);
  dlf.assign(Ntot + 1, 0.);
  dlfi.assign(Ntot + 1, 0.);
  dlvi.assign(Ntot + 1, 0.);
  for (int i = 0; i < Ntot; ++i) {
    dlf[i] = lf[i + 1] - lf[i];
    dlfi[i] = 1. / dlf[i];
    lv[i] = 0.5 * (lf[i] + lf[i + 1]);
  }
  for (int i = 1; i < Ntot; ++i) {
    double dlv = lv[i] - lv[i - 1];
    dlvi[i] = 1. / dlv;
  }
}

// Tile lists of the default fused variant (predictor tiles cover cells
// 1..Ntot-2, corrector tiles the active cells).
void tiles_of(int N0, int N1, int ng, bool pred, int tx, int ty, std::vector<FusedTile>& out) {
  const int T[2] = {tx, ty};
  const int N[2] = {N0, N1};
  int nt[2];
  for (int a = 0; a < 2; ++a) nt[a] = (N[a] + T[a] - 1) / T[a];
  for (int by = 0; by < nt[1]; ++by)
    for (int bx = 0; bx < nt[0]; ++bx) {
      int lo[2], hi[2];
      const int t[2] = {bx, by};
      for (int a = 0; a < 2; ++a) {
        lo[a] = ng + t[a] * T[a];
        hi[a] = std::min(ng + (t[a] + 1) * T[a], ng + N[a]) - 1;
        if (pred) {
          if (t[a] == 0) lo[a] = 1;
          if (t[a] == nt[a] - 1) hi[a] = N[a] + 2 * ng - 2;
        }
      }
      out.push_back(FusedTile{0, lo[0], lo[1], hi[0] - lo[0] + 1, hi[1] - lo[1] + 1});
    }
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
  for (int a = 0; a < 2; ++a) {
    if (!(g->lmax[a] > g->lmin[a])) return fail(BNZ_ERR_ARG, "lmax must exceed lmin");
    for (int sd = 0; sd < 2; ++sd)
      if (g->bc[a][sd] < 0 || g->bc[a][sd] > 2) return fail(BNZ_ERR_ARG, "bc flag must be 0, 1 or 2");
    if ((g->bc[a][0] == BNZ_BC_PERIODIC) != (g->bc[a][1] == BNZ_BC_PERIODIC))
      return fail(BNZ_ERR_ARG, "periodic boundaries must be set on both sides of an axis");
  }
  const int nx = g->Nx + 2 * ng, ny = g->Ny + 2 * ng;
  const size_t ncell = (size_t)nx * ny;
  const FusedVariant& v = FUSED_VARIANTS[0];
  std::vector<FusedTile> tiles;
  tiles_of(g->Nx, g->Ny, ng, true, v.tx, v.ty, tiles);
  const int ntA = (int)tiles.size();
  tiles_of(g->Nx, g->Ny, ng, false, v.tx, v.ty, tiles);
  const int ntB = (int)tiles.size() - ntA;
  // layout of the scratch array
  const size_t o_inst = 0;
  const size_t o_ds = align256(o_inst + sizeof(FusedInst));
  const size_t o_err = align256(o_ds + sizeof(DtState));
  const size_t o_tiles = align256(o_err + sizeof(unsigned));
  const size_t o_coord = align256(o_tiles + tiles.size() * sizeof(FusedTile));
  const size_t ncoord = 5 * (size_t)(nx + 1) + 5 * (size_t)(ny + 1) + 5 * 2;
  const size_t o_ws = align256(o_coord + ncoord * sizeof(double));
  const size_t o_bs = align256(o_ws + 9 * ncell * sizeof(double));
  const size_t need = align256(o_bs + 3 * ncell * sizeof(double));
  if (need > kScratchBytes)
    return fail(BNZ_ERR_ARG, "grid too large for the no-alloc step: it needs " + std::to_string(need) +
                                 " bytes of scratch and the fixed array holds " + std::to_string(kScratchBytes) +
                                 " ((Nx+6)*(Ny+6) must stay below about 40000 cells)");
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;

  // coordinates (x, y, and the single z cell), 5 arrays per axis
  std::vector<double> host(ncoord, 0.);
  const double* dcoord = reinterpret_cast<const double*>(base + o_coord);
  const double* ptr[3][5];
  {
    size_t off = 0;
    const int N[3] = {nx, ny, 1};
    const int i1[3] = {ng, ng, 0}, i2[3] = {ng + g->Nx - 1, ng + g->Ny - 1, 0};
    for (int a = 0; a < 3; ++a) {
      std::vector<double> lf, lv, dlf, dlfi, dlvi;
      axis_coords(a, N[a], i1[a], i2[a], g, lf, lv, dlf, dlfi, dlvi);
      const std::vector<double>* arr[5] = {&dlf, &dlfi, &lf, &lv, &dlvi};
      const size_t len = (size_t)N[a] + 1;
      for (int q = 0; q < 5; ++q) {
        for (size_t k = 0; k < len; ++k) host[off + k] = (*arr[q])[k];
        ptr[a][q] = dcoord + off;
        off += len;
      }
    }
  }
  FusedInst I;
  memset(&I, 0, sizeof I);
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
  // the time record and the error word start from zero on every call: the
  // array keeps whatever the previous call left in it
  DtState ds;
  memset(&ds, 0, sizeof ds);
  ds.dt = dt;
  ds.tmax = 1e300;
  unsigned zero = 0;
  cudaError_t e;
  e = cudaMemcpyAsync(base + o_inst, &I, sizeof I, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_ds, &ds, sizeof ds, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_err, &zero, sizeof zero, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + o_tiles, tiles.data(), tiles.size() * sizeof(FusedTile), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(base + o_coord, host.data(), ncoord * sizeof(double), cudaMemcpyHostToDevice, s);
  // the host copies above must land before the host buffers go out of scope
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(BNZ_ERR_CUDA, std::string("scratch upload: ") + cudaGetErrorString(e));

  const Launchers* L = m->exact_fp ? &exact::table : &fast::table;
  FusedLaunch f;
  memset(&f, 0, sizeof f);
  f.insts = reinterpret_cast<const FusedInst*>(base + o_inst);
  f.ninst = 1;
  f.tilesA = reinterpret_cast<const FusedTile*>(base + o_tiles);
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
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BNZ_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return BNZ_OK;
}

const char* bnz_noalloc_last_error(void) { return g_err.c_str(); }

size_t bnz_noalloc_scratch_bytes(void) { return kScratchBytes; }

}  // extern "C"
