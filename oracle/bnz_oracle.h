/*
 * bnz_oracle.h -- CPU ORACLE for the VL2 + HLL/HLLT/HLLD + CT step of bonzo.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker / the timed CPU reference.
 *
 * It is a plain-C restatement of the reference's algorithm:
 *   - the C kernels of src/mhd/eos_c.{c,h}, src/mhd/fluxes_c.c and
 *     src/coordinates/reconstr_c.{c,h} (restated point by point, same
 *     arithmetic order, pinned bitwise against the reference's own compiled
 *     kernels by tests/test_oracle_kernels.py);
 *   - the Cython orchestration that cannot be built as shipped:
 *     src/integration/{vanleer,godunov,ct,new_dt,integrator}.pyx,
 *     src/bc/{grid_bc,grid_bc_funcs,util_bc}.pyx,
 *     src/dissipation/{diffusion,thcond_elec,util_diffusion}.pyx.
 *
 * Kernels use the reference's row-pointer ABI (real** rows, i1..i2 ranges)
 * so that the driver can run either the restated kernels or the reference's
 * compiled ones (oracle/_ref/libbnzref.so) through the same call sites.
 */
#ifndef BNZ_ORACLE_H
#define BNZ_ORACLE_H

#include <stdint.h>

typedef double real;

#ifndef ORC_MFIELD
#define ORC_MFIELD 1
#endif

/* Variable layout: src/defs_c.h:68-85 (MFIELD, no CGL/TWOTEMP). */
#if ORC_MFIELD
#define ORC_NMODE 9
#define ORC_NVAR 12
enum { O_RHO = 0, O_MX, O_MY, O_MZ, O_EN, O_PSC, O_BX, O_BY, O_BZ };
#else
#define ORC_NMODE 6
#define ORC_NVAR 6
enum { O_RHO = 0, O_MX, O_MY, O_MZ, O_EN, O_PSC };
#endif
enum { O_VX = 1, O_VY = 2, O_VZ = 3, O_PR = 4 };

/*
 * Coordinate block with the member order and types of the reference's
 * GridCoord (src/coordinates/coord_c.h:19-99, with the missing ';' after
 * interp_order restored).  The layout has to match because the driver can
 * hand this struct to the reference's compiled reconstr_const /
 * reconstr_linear, which read lf, lv, dlv, dlv_inv, scale and geom from it.
 */
typedef struct {
  int Nact[3];
  int Ntot[3];
  int Nact_glob[3];
  int Ntot_glob[3];
  int ng;
  int i1, i2;
  int j1, j2;
  int k1, k2;
  real lmin[3];
  real lmax[3];
  real **lf;
  real **lv;
  real **dlf;
  real **dlv;
  real **dlf_inv;
  real **dlv_inv;
  int geom;      /* CoordGeom: 0 = Cartesian */
  int scale[3];  /* CoordScale: 0 = uniform */
  int interp_order;
  int rank;
  int pos[3];
  int size[3];
  int size_tot;
  int ***ranks;
  int nbr_ranks[3][2];
  real *syxf;
  real *syxv;
  real *szxf;
  real *szxv;
  real *szyf;
  real *szyv;
  real *rinv_mean;
  real *d2r;
  real *d3r;
  real *sin_thf;
  real *sin_thv;
  real *dcos_thf;
  real *src_coeff1;
  real **src_coeff2;
} orc_coord;

/* Row-pointer kernel ABI (src/mhd/fluxes_c.h:3-20, src/coordinates/reconstr_c.h:4-12). */
typedef void (*orc_rsolver_fn)(real **flux, real **wl, real **wr, real *bx,
                               int i1, int i2, real gam);
typedef void (*orc_reconstr_fn)(real **wl, real **wr, real ***w, real ***scr,
                                orc_coord *gc, int ax, int i1, int i2, int j,
                                int k, int char_proj, real gam);
typedef void (*orc_row_eos_fn)(real **out, real **in, int i1, int i2, real gam);

/* Method enums (src/integration/integrator.pxd:52-91 names). */
enum { ORC_RS_HLL = 0, ORC_RS_HLLC = 1, ORC_RS_HLLD = 2, ORC_RS_HLLT = 3 };
enum { ORC_RCN_CONST = 0, ORC_RCN_LINEAR = 1 };
enum { ORC_LIM_VL = 0, ORC_LIM_MC = 1, ORC_LIM_MM = 2 };
enum { ORC_BC_PERIODIC = 0, ORC_BC_OUTFLOW = 1, ORC_BC_REFLECT = 2 };
enum { ORC_TC_ISO = 0, ORC_TC_ANISO = 1 };

typedef struct {
  int Nx, Ny, Nz;       /* active cells per axis (Ny/Nz = 1 below 2D/3D) */
  int dims;             /* 1, 2 or 3: the reference's D2D / D3D build flags */
  real lmin[3], lmax[3];
  int bc[3][2];         /* bc_x1.. bc_z2 flags */
  real gam, cour;
  int rsolver, reconstr, limiter, charact_proj;
  real kappa0;          /* 0 switches conduction off */
  int thcond_type;      /* ORC_TC_ISO / ORC_TC_ANISO */
  int sat_hfe;
  real cour_diff;
  int fixdt;            /* FIXDT build flag */
  real dt_fixed;
  int outflow_face_aware; /* 1: outflow keeps the CT-updated outer face */
  int nthreads;         /* OpenMP threads (0: library default) */
  int rows_parallel;    /* 0: reference threading (prange over k / j only) */
  /* source terms (src/srcterms): constant gravity and turbulence driving */
  real grav[3];         /* gx, gy, gz (gravity.pyx:17-19) */
  real drive_f0;        /* driving amplitude f0 (turb_driv.pyx:27), 0 = off */
  real drive_tau;       /* correlation time tau */
  int drive_nmod;       /* modes per axis nmod */
  uint64_t drive_seed;  /* seed of the mode amplitudes (splitmix64) */
} orc_params;

typedef struct orc_sim orc_sim;

/* Lifecycle ------------------------------------------------------------- */
orc_sim *orc_create(const orc_params *p);
void orc_destroy(orc_sim *s);
int orc_ntot(const orc_sim *s, int ax);
int orc_ng(const orc_sim *s);
/* Address of the simulation's GridCoord-compatible coordinate block. */
void *orc_coord_block(orc_sim *s);
/* Run a row-ABI reconstruction function (restated or the reference's) on one
 * row w (NMODE, n): cells 1..n-2, wl/wr (NMODE, n+1), axis x. */
void orc_reconstr_flat_with(orc_reconstr_fn fn, int order, int char_proj, real *wl, real *wr,
                            const real *w, int n, real gam, void *gc);
/* Coordinates (lf has Ntot+1 entries, the others Ntot). */
void orc_get_coord(const orc_sim *s, int ax, real *lf, real *lv, real *dlf);

/* Swap in the reference's own compiled kernels (NULL keeps the restated one). */
void orc_set_kernels(orc_sim *s, orc_rsolver_fn rs, orc_reconstr_fn rc_const,
                     orc_reconstr_fn rc_linear);

/* State: full arrays including ghosts, layout (NMODE|3, Nz, Ny, Nx) C-order. */
void orc_set_state(orc_sim *s, const real *prim, const real *bfld);
void orc_get_state(const orc_sim *s, real *prim, real *cons, real *bfld);
/* init_sim steps after set_problem (src/integration/vanleer.pyx:41-48). */
void orc_init(orc_sim *s);

/* Step pieces ----------------------------------------------------------- */
real orc_new_dt(orc_sim *s);
void orc_vl2_step(orc_sim *s, real dt);   /* vanleer.pyx:101-163 */
void orc_diffuse(orc_sim *s, real dt);    /* thcond_elec.pyx:17-113 */
void orc_apply_bc(orc_sim *s, uint32_t var_mask);
/* vanleer.advance: loop until time >= tmax or max_steps reached. */
void orc_advance(orc_sim *s, real tmax, int max_steps);
real orc_time(const orc_sim *s);
long orc_step_count(const orc_sim *s);
real orc_last_dt(const orc_sim *s);
int orc_last_nsts(const orc_sim *s);

/* Exposed restated kernels (for the pinning tests) ----------------------- */
void orc_hll_flux(real **flux, real **wl, real **wr, real *bx, int i1, int i2, real gam);
void orc_hllt_flux(real **flux, real **wl, real **wr, real *bx, int i1, int i2, real gam);
#if ORC_MFIELD
void orc_hlld_flux(real **flux, real **wl, real **wr, real *bx, int i1, int i2, real gam);
#else
void orc_hllc_flux(real **flux, real **wl, real **wr, real *bx, int i1, int i2, real gam);
#endif
void orc_cons2prim_1(real **w1, real **u1, int i1, int i2, real gam);
void orc_prim2cons_1(real **u1, real **w1, int i1, int i2, real gam);
real orc_fms(real *w, real bx, real gam);
void orc_reconstr_const(real **wl, real **wr, real ***w, real ***scr, orc_coord *gc,
                        int ax, int i1, int i2, int j, int k, int char_proj, real gam);
void orc_reconstr_linear(real **wl, real **wr, real ***w, real ***scr, orc_coord *gc,
                         int ax, int i1, int i2, int j, int k, int char_proj, real gam);
void orc_reconstr_linear_mc(real **wl, real **wr, real ***w, real ***scr, orc_coord *gc,
                            int ax, int i1, int i2, int j, int k, int char_proj, real gam);
void orc_reconstr_linear_mm(real **wl, real **wr, real ***w, real ***scr, orc_coord *gc,
                            int ax, int i1, int i2, int j, int k, int char_proj, real gam);
/* Flat-array conveniences for tests: n points, arrays (NMODE, n). */
void orc_flux_flat(int rsolver, real *flux, const real *wl, const real *wr,
                   const real *bx, int n, real gam);
void orc_reconstr_flat(int reconstr, int limiter, int char_proj, real *wl,
                       real *wr, const real *w, int n, real gam);
/* RKL2 coefficients (diffusion.pyx:217-260); coeff has (s+1)*4 entries. */
int orc_get_nsts(real dt_hyp, real dt_diff);
void orc_get_sts_coeff(int s, real *coeff);
#endif
