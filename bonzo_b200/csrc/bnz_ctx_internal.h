// bnz_ctx_internal.h -- the context structure behind the opaque bnz_ctx of
// the C ABI, and the host helpers shared by the translation units that
// implement the ABI (bnz_ctx.cu, bnz_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/bnz_gpu.h"
#include "bnz_common.h"
#include "bnz_launch.h"

struct bnz_ctx {
  bnz_grid_desc gd;
  bnz_method_desc md;
  int Ntot[3];
  int ng;
  int i1, i2, j1, j2, k1, k2;
  size_t ncell;
  std::vector<double> lf[3], lv[3], dlf[3], dlf_inv[3], dlv[3], dlv_inv[3];
  double* d_coord = nullptr;
  GridDev g;
  // state and scratch
  double* prim = nullptr;
  double* cons = nullptr;
  double* bfld = nullptr;
  double* cons_s = nullptr;
  double* bfld_s = nullptr;
  double* flx[3] = {nullptr, nullptr, nullptr};
  double* ec = nullptr;
  double* ee = nullptr;
  double* wnext = nullptr;
  double* bnext = nullptr;
  // fused path: ping-pong state buffers, tile lists, instance descriptor
  double* wbuf[2] = {nullptr, nullptr};
  double* bbuf[2] = {nullptr, nullptr};
  int parity = 0;
  bool ghosts_stale = false;  // fused path: ghosts / cons not refreshed since the last step
  bool cons_stale = false;    // split path: cons not formed from prim since the last step
  FusedInst* d_inst = nullptr;
  FusedTile* d_tiles = nullptr;
  int ntA = 0, ntB = 0;
  // fused 3D path: instance record, chunk lists (predictor then corrector),
  // the 4D tensor map of ws (null when Ntot_x is odd)
  FusedInst3* d_inst3 = nullptr;
  FusedTile3* d_tiles3 = nullptr;
  int ntA3 = 0, ntB3 = 0;
  unsigned char* d_map3 = nullptr;
  unsigned char* d_smaps = nullptr;  // split path, 3D: the update kernel's tensor maps
  int graph_parity = -1;
  int variant = 0;
  // conduction scratch
  double* dscr = nullptr;
  DiffArgs da;
  int last_nsts = 0;
  // device scalars
  unsigned* d_err = nullptr;
  DtState* d_ds = nullptr;
  double* d_sts = nullptr;  // stage coefficients (4 per stage)
  int sts_cap = 0;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  double graph_tmax = -1.;
  const Launchers* L = nullptr;
  std::string err;
  double time = 0.;
  long step = 0;
  double last_dt = 0.;
  long long launches = 0;  // kernels launched through this context
  long long graph_launches = 0;
  double h_stage[3] = {0., 0., 0.};  // host staging for async copies of the time record
  long long h_step = 0;
  bool time_on_device = false;  // the device DtState holds the current time
  bool own_stream = true;
  struct bnz_adj* adj = nullptr;  // adjoint tape (bnz_adjoint.cu), created on first use
  struct bnz_io* io = nullptr;    // history / snapshot resources (bnz_io.cu), created on first use
  // turbulence driving: force field, this step's mode amplitudes (device and
  // pinned staging, guarded by an event), the amplitude stream's state
  double* fdriv = nullptr;
  double* d_modes = nullptr;
  double* h_modes = nullptr;
  cudaEvent_t ev_modes = nullptr;
  unsigned long long rng = 0;
};

namespace bnzi {

// record msg as the context's last error and return code
int fail(bnz_ctx* c, int code, const std::string& msg);
StepArgs step_args(bnz_ctx* c);
FusedInst make_inst(const bnz_ctx* c);
FusedLaunch fused_launch(const bnz_ctx* c, int dt_mode);
FusedInst3 make_inst3(const bnz_ctx* c);
Fused3Launch fused3_launch(const bnz_ctx* c, int dt_mode);
// chunk lists of a 3D grid: the predictor range (cells 1..Ntot-2) or the
// active cells, in chunks of at most tx x ty cells and about kz planes
void make_tiles3(int inst, const int* N, int ng, bool pred, int tx, int ty, int kz, std::vector<FusedTile3>& out);
// the 4D tensor map (x, y, z, field) of a 9-field array of the context for
// the 3D corrector's staging box; false when Ntot_x is odd or the driver
// entry point is missing
bool ws_map3(const bnz_ctx* c, const double* base, void* map128);
cudaError_t build_split_maps(bnz_ctx* c);
bool fused_available(const bnz_grid_desc* g, const bnz_method_desc* m);
void set_parity(bnz_ctx* c, int p);
int ensure_ghosts(bnz_ctx* c);
int refresh_cds(bnz_ctx* c);
// vanleer.pyx:101-163 with dt taken as dt_mode says (FDT_EXPLICIT: d_ds->dt)
int step_impl(bnz_ctx* c, double dt_host, int dt_mode = FDT_EXPLICIT);
// sources on: gravity or driving
bool src_on(const bnz_method_desc& m);
bool drive_on(const bnz_method_desc& m);
// release the adjoint tape (bnz_adjoint.cu) and the output resources (bnz_io.cu)
void adj_free(bnz_ctx* c);
void io_free(bnz_ctx* c);

}  // namespace bnzi

#define CKC(call)                                                                                \
  do {                                                                                           \
    cudaError_t _e = (call);                                                                     \
    if (_e != cudaSuccess)                                                                       \
      return bnzi::fail(c, BNZ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));   \
  } while (0)
