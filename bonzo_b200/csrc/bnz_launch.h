// bnz_launch.h -- host launchers of one floating-point mode, and the dispatch
// table the context uses to pick the exact (no contraction) or fast build.
#pragma once

#include "bnz_common.h"

struct Launchers {
  int (*plain_predictor_corrector)(const StepArgs&, const double* dtp);
  int (*fused_step)(const FusedLaunch&, int parity);
  int (*fused_time)(const FusedLaunch&);
  int (*fused_cds)(const FusedLaunch&, int parity);
  int (*apply_bc)(const StepArgs&, double* prim, double* bfld, unsigned mask);
  int (*prim2cons_all)(const StepArgs&);
  int (*cons2prim_all)(const StepArgs&);
  int (*interp_bc_active)(const StepArgs&);
  int (*new_dt)(const StepArgs&, const double* prim, DtState* ds, double cour, int clip);
  int (*set_dt)(cudaStream_t, DtState*, double);
  int (*time_advance)(cudaStream_t, DtState*);
  int (*diff_dt_max)(const StepArgs&, const DiffArgs&, unsigned long long* slot);
  int (*diff_stage)(const StepArgs&, const DiffArgs&, int first, const double* coef, const double* dtp);
  int (*adj_step)(const FusedInst& I, const AdjStep& s);
  int (*source)(const StepArgs&, double* u1, const double* w0, int order, const double* dtp, double fac);
  int (*drive)(const StepArgs&, const DriveArgs&, const double* dtp);
  int (*riemann_rows)(int rs, const double* wl, const double* wr, const double* bx, double* flux, int n, int nvar,
                      double gam, unsigned* err, cudaStream_t s);
  int (*fused3_step)(const Fused3Launch&, int parity);
  int (*fused3_time)(const Fused3Launch&);
  int (*fused3_cds)(const Fused3Launch&, int parity);
  int (*split_predictor_corrector)(const StepArgs&, const double* dtp);
  int (*fixed_dt)(cudaStream_t, DtState*, double);
};

#define BNZ_DECLARE_LAUNCHERS(NS)                                                                     \
  namespace NS {                                                                                      \
  int plain_predictor_corrector(const StepArgs&, const double* dtp);                                \
  int fused_step(const FusedLaunch&, int parity);                                                    \
  int fused_time(const FusedLaunch&);                                                                 \
  int fused_cds(const FusedLaunch&, int parity);                                                      \
  int apply_bc(const StepArgs&, double* prim, double* bfld, unsigned mask);                         \
  int prim2cons_all(const StepArgs&);                                                                \
  int cons2prim_all(const StepArgs&);                                                                \
  int interp_bc_active(const StepArgs&);                                                             \
  int new_dt(const StepArgs&, const double* prim, DtState* ds, double cour, int clip);              \
  int set_dt(cudaStream_t, DtState*, double);                                                        \
  int time_advance(cudaStream_t, DtState*);                                                          \
  int diff_dt_max(const StepArgs&, const DiffArgs&, unsigned long long* slot);                      \
  int diff_stage(const StepArgs&, const DiffArgs&, int first, const double* coef, const double* dtp);  \
  int adj_step(const FusedInst& I, const AdjStep& s);                                                \
  int source(const StepArgs&, double* u1, const double* w0, int order, const double* dtp, double fac);  \
  int drive(const StepArgs&, const DriveArgs&, const double* dtp);                                    \
  int riemann_rows(int rs, const double* wl, const double* wr, const double* bx, double* flux, int n, int nvar, \
                   double gam, unsigned* err, cudaStream_t s);                                          \
  int fused3_step(const Fused3Launch&, int parity);                                                  \
  int fused3_time(const Fused3Launch&);                                                               \
  int fused3_cds(const Fused3Launch&, int parity);                                                    \
  int split_predictor_corrector(const StepArgs&, const double* dtp);                                \
  int fixed_dt(cudaStream_t, DtState*, double);                                                      \
  extern const Launchers table;                                                                       \
  }

BNZ_DECLARE_LAUNCHERS(exact)
BNZ_DECLARE_LAUNCHERS(fast)

#define BNZ_DEFINE_TABLE(NS)                                                                          \
  const Launchers NS::table = {NS::plain_predictor_corrector, NS::fused_step, NS::fused_time,       \
                               NS::fused_cds, NS::apply_bc,                                           \
                               NS::prim2cons_all, NS::cons2prim_all, NS::interp_bc_active,           \
                               NS::new_dt, NS::set_dt, NS::time_advance, NS::diff_dt_max,            \
                               NS::diff_stage, NS::adj_step, NS::source,    \
                               NS::drive, NS::riemann_rows, NS::fused3_step, NS::fused3_time,        \
                               NS::fused3_cds, NS::split_predictor_corrector, NS::fixed_dt};
