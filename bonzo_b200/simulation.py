"""Python-level facade with the reference's names: Simulation(usr_dir),
.advance(tmax), .prim / .cons / .bfld, over one device context.

It mirrors the reference's top level:
  - Simulation (src/simulation.pyx:55-86): builds the grid, the integrator and
    the I/O from usr_dir/config.cfg, sets the problem (or restarts), then
    advance(tmax) steps to tmax;
  - BnzGrid / BnzIntegr: the host-side grid (GridCoord, prim / cons / bfld
    arrays with ghosts, src/coordinates/grid.pyx:30-52) and the method and
    time record (src/integration/integrator.pxd:97-187), filled from the
    config keys the reference reads (bonzo_b200.config.read_param);
  - init (src/integration/vanleer.pyx:20-56): problem generator
    set_problem(grid, integr, usr_dir) writing prim and face B on the active
    cells, then ghost fill, cell B from the faces and cons on the device;
  - advance (vanleer.pyx:59-179): one CFL step at a time on the device (dt
    clipped to tmax), after each step the output schedule of BnzIO
    (src/io/io.pyx:124-236): history row, full grid, slice and restart files
    whenever the time crosses a multiple of their interval.

Output formats follow src/io/output.pyx:248-430 with numpy .npz in place of
HDF5 (h5py is not available): datasets rho, vx, vy, vz, p, psc (or rho, mx,
my, mz, en, psc with variable_type cons), bxc, byc, bzc, bxf, byf, bzf in the
(Nz, Ny, Nx) layout, with or without ghosts, plus entries time, step, dt, xf,
yf, zf for the file attributes.  The history file out/hst.txt has the
reference's column names and '{:<14e}' format.  Grid files are written from
an asynchronous device->host snapshot by a background thread, so stepping
continues while the previous output drains.
"""
import importlib.util
import os
import threading

import numpy as np

from . import config as cfg
from . import problems
from ._lib import Context
from .coords import GridCoord

HST_NAMES = ['[0]step', '[1]time', '[2]<rho_gas>', '[3]<Ek_gas>', '[4]<Eth_gas>',
             '[5]<Em_gas>', '[6]<Etot>', '[7]<vx_gas>', '[8]<vy_gas>', '[9]<vz_gas>',
             '[10]<Bx>', '[11]<By>', '[12]<Bz>', '[13]rms(Bx)', '[14]rms(By)', '[15]rms(Bz)']
PRIM_NAMES = ['rho', 'vx', 'vy', 'vz', 'p', 'psc']
CONS_NAMES = ['rho', 'mx', 'my', 'mz', 'en', 'psc']
B_NAMES = ['bxc', 'byc', 'bzc', 'bxf', 'byf', 'bzf']


def _pinned(shape):
    """Page-locked host array when torch is importable (true copy overlap)."""
    try:
        import torch
        if torch.cuda.is_available():
            return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        pass
    return np.empty(shape)


class BnzGrid:
    """Grid coordinates and host copies of the state (GridData names)."""

    def __init__(self, usr_dir):
        rp = lambda s, k, t: cfg.read_param(s, k, t, usr_dir)
        N = [rp("computation", "Nx", "i"), rp("computation", "Ny", "i"), rp("computation", "Nz", "i")]
        dims = 3 if N[2] > 1 else 2 if N[1] > 1 else 1
        lmin = [rp("computation", k, "f") for k in ("xmin", "ymin", "zmin")]
        lmax = [rp("computation", k, "f") for k in ("xmax", "ymax", "zmax")]
        bc = [[rp("physics", "bc_%s%d" % (a, s), "i") for s in (1, 2)] for a in "xyz"]
        for a in range(3):
            for s in range(2):
                if bc[a][s] not in (0, 1, 2):
                    raise cfg.ConfigError("bc flag %d on axis %d is not supported (0, 1, 2)" % (bc[a][s], a))
        reconstr = rp("computation", "reconstr", "s")
        ng = 2 if reconstr == "const" else 3
        self.usr_dir = usr_dir
        self.dims = dims
        self.bc = tuple(tuple(b) for b in bc)
        self.coord = GridCoord(N[0], N[1], N[2], dims, lmin, lmax, self.bc, ng)
        shape = tuple(self.coord.Ntot[::-1])
        self.prim = np.zeros((9,) + shape)
        self.cons = np.zeros((9,) + shape)
        self.bfld = np.zeros((3,) + shape)


class BnzIntegr:
    """Method parameters and the time record (the integrator's fields)."""

    def __init__(self, coord, usr_dir):
        rp = lambda s, k, t: cfg.read_param(s, k, t, usr_dir)
        self.gam = rp("physics", "gam", "f")
        self.cour = rp("computation", "cour", "f")
        self.cour_diff = rp("computation", "cour_diff", "f")
        self.rsolver = rp("computation", "rsolver", "s")
        self.reconstr = rp("computation", "reconstr", "s")
        self.limiter = rp("computation", "limiter", "s")
        self.char_proj = rp("computation", "charact_proj", "i")
        self.kappa0 = rp("physics", "kappa0", "f")
        self.thcond_type = rp("physics", "elec_thcond_type", "s")
        self.sat_hfe = rp("physics", "sat_hfe", "i")
        self.tmax = rp("computation", "tmax", "f")
        # source terms (gravity.pyx:17-19 gx/gy/gz; the shipped config's g0 is
        # "constant negative g along Y"; turb_driv.pyx:27-29 f0/tau/nmod)
        rd = lambda s_, k, t, d: cfg.read_param(s_, k, t, usr_dir, d)
        g0 = rd("physics", "g0", "f", 0.0)
        self.grav = (rd("physics", "gx", "f", 0.0), rd("physics", "gy", "f", -g0), rd("physics", "gz", "f", 0.0))
        self.drive_f0 = rd("physics", "f0", "f", 0.0)
        self.drive_tau = rd("physics", "tau", "f", 1.0) or 1.0
        self.drive_nmod = rd("physics", "nmod", "i", 1)
        self.drive_seed = rd("physics", "driving_seed", "i", 0)
        self.time = 0.0
        self.step = 0
        self.dt = 0.0

    def method(self):
        return dict(gam=self.gam, cour=self.cour, rsolver=self.rsolver, reconstr=self.reconstr,
                    limiter=self.limiter, charact_proj=self.char_proj, kappa0=self.kappa0,
                    thcond_type=self.thcond_type, sat_hfe=self.sat_hfe, cour_diff=self.cour_diff,
                    grav=self.grav, drive_f0=self.drive_f0, drive_tau=self.drive_tau,
                    drive_nmod=self.drive_nmod, drive_seed=self.drive_seed)


class BnzIO:
    """Output schedule and writers (src/io/io.pyx)."""

    def __init__(self, usr_dir):
        rp = lambda s, k, t, d=None: cfg.read_param(s, k, t, usr_dir, d)
        self.usr_dir = usr_dir
        self.hst_dt = rp("output", "history_dt", "f", 0.0)
        self.grid_dt = rp("output", "grid_dt", "f", 0.0)
        self.slc_dt = rp("output", "slice_dt", "f", 0.0)
        self.rst_dt = rp("restart", "restart_dt", "f", 0.0)
        self.restart = rp("restart", "restart", "i", 0)
        self.var_type = rp("output", "variable_type", "s", "prim")
        self.write_ghost = rp("output", "write_ghost_cells", "i", 0)
        self.slc_axis = "xyz".index(rp("output", "slice_axis", "s", "z"))
        self.slc_loc = rp("output", "slice_cell_index", "i", 0)
        self.out_dir = os.path.join(usr_dir, "out")
        self.rst_dir = os.path.join(usr_dir, "rst")
        self._writer = None
        self._bufs = None
        if not self.restart:
            os.makedirs(self.out_dir, exist_ok=True)
            os.makedirs(self.rst_dir, exist_ok=True)
            with open(os.path.join(self.out_dir, "hst.txt"), "w") as f:
                f.write("".join("{:<14}".format(n) for n in HST_NAMES) + "\n")

    @staticmethod
    def _due(time, dt, every):
        # io.pyx:137-140: write when the step crossed a multiple of `every`
        if every == 0.0:
            return False
        t1 = int(time / every) * every
        return time - dt < t1 <= time

    def write_output(self, sim):
        integr = sim.integr
        dt = integr.dt if integr.time > 0.0 else 1e-6
        if self._due(integr.time, dt, self.hst_dt):
            self.write_history(sim)
        if self._due(integr.time, dt, self.grid_dt):
            self.write_grid(sim, rst=False)
        if self._due(integr.time, dt, self.slc_dt):
            self.write_grid(sim, rst=False, slice_only=True)

    def write_restart(self, sim):
        integr = sim.integr
        if self._due(integr.time, integr.dt, self.rst_dt):
            self.write_grid(sim, rst=True)

    def write_history(self, sim):
        row = sim.ctx.history()
        with open(os.path.join(self.out_dir, "hst.txt"), "a") as f:
            f.write("".join("{:<14e}".format(v) for v in row) + "\n")

    def _snapshot(self, sim):
        if self._writer is not None:
            self._writer.join()
        if self._bufs is None:
            shape = sim.ctx.shape
            self._bufs = (_pinned((9,) + shape), _pinned((9,) + shape), _pinned((3,) + shape))
        P, U, B = self._bufs
        sim.ctx.snapshot(P, U, B)
        return P, U, B

    def write_grid(self, sim, rst=False, slice_only=False):
        """output.pyx:248-400 write_grid (and write_slice with slice_only)."""
        gc = sim.grid.coord
        integr = sim.integr
        P, U, B = self._snapshot(sim)
        ghost = self.write_ghost and not rst
        cons = self.var_type == "cons" and not rst
        if rst:
            path = os.path.join(self.rst_dir, "rst_grid.npz")
        elif slice_only:
            path = os.path.join(self.out_dir, "slice_{:03d}.npz".format(int(integr.time / self.slc_dt)))
        else:
            path = os.path.join(self.out_dir, "grid_{:03d}.npz".format(int(integr.time / self.grid_dt)))
        if ghost:
            sl = np.s_[:, :, :]
        else:
            sl = np.s_[gc.k1:gc.k2 + 1, gc.j1:gc.j2 + 1, gc.i1:gc.i2 + 1]
        attrs = dict(time=integr.time, step=integr.step, dt=integr.dt,
                     xf=np.asarray(gc.lf[0]), yf=np.asarray(gc.lf[1]), zf=np.asarray(gc.lf[2]))
        names = (CONS_NAMES if cons else PRIM_NAMES) + B_NAMES
        axis, loc = self.slc_axis, self.slc_loc

        def work():
            sim.ctx.snapshot_wait()
            src = U if cons else P
            data = {}
            for n in range(6):
                data[names[n]] = src[n][sl]
            for n in range(3):
                data[names[6 + n]] = src[6 + n][sl]
                data[names[9 + n]] = B[n][sl]
            if slice_only:
                # the slice through cell index loc of the written range, normal to `axis`
                data = {k: np.take(v, loc, axis=2 - axis) for k, v in data.items()}
            np.savez(path, **data, **attrs)

        self._writer = threading.Thread(target=work, daemon=True)
        self._writer.start()

    def flush(self):
        if self._writer is not None:
            self._writer.join()
            self._writer = None

    def set_restart(self, grid, integr):
        """restart.pyx:23-117: active prim and face B, time and step."""
        gc = grid.coord
        with np.load(os.path.join(self.rst_dir, "rst_grid.npz")) as f:
            sl = np.s_[gc.k1:gc.k2 + 1, gc.j1:gc.j2 + 1, gc.i1:gc.i2 + 1]
            for n in range(6):
                grid.prim[n][sl] = f[PRIM_NAMES[n]]
            for n in range(3):
                grid.prim[6 + n][sl] = f[B_NAMES[n]]
                grid.bfld[n][sl] = f[B_NAMES[3 + n]]
            # the outer faces the CT update owns (face i2+1, j2+1, k2+1) come
            # back through the boundary fill after init
            integr.time = float(f["time"])
            integr.step = int(f["step"])


def _load_problem(problem, usr_dir):
    """A set_problem(grid, integr, usr_dir) callable: given directly, a name of
    bonzo_b200.problems.SET_PROBLEM, the [problem] name key, or usr_dir/problem.py."""
    if callable(problem):
        return problem
    name = problem or cfg.read_param("problem", "name", "s", usr_dir, "")
    if name:
        if name not in problems.SET_PROBLEM:
            raise cfg.ConfigError("unknown problem %r (known: %s)" % (name, ", ".join(sorted(problems.SET_PROBLEM))))
        return problems.SET_PROBLEM[name]
    path = os.path.join(usr_dir, "problem.py")
    if not os.path.exists(path):
        raise cfg.ConfigError("no problem given: pass problem=, set [problem] name, or provide %s" % path)
    spec = importlib.util.spec_from_file_location("bnz_user_problem", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.set_problem


class Simulation:
    """src/simulation.pyx:55-86 over the device context."""

    def __init__(self, usr_dir, problem=None, path="fused", exact_fp=False):
        self.usr_dir = usr_dir
        self.grid = BnzGrid(usr_dir)
        self.integr = BnzIntegr(self.grid.coord, usr_dir)
        self.io = BnzIO(usr_dir)
        gc = self.grid.coord
        if path == "fused" and not (gc.dims == 2 and self.integr.reconstr == "linear"):
            # the fused tile kernels are the fastest on 2D PLM grids, the split
            # path (fluxes once per face, one update per stage) elsewhere
            path = "split"
        self.ctx = Context(Nx=gc.Nact[0], Ny=gc.Nact[1], Nz=gc.Nact[2], dims=gc.dims, lmin=gc.lmin,
                           lmax=gc.lmax, bc=self.grid.bc, path=path, exact_fp=int(exact_fp),
                           **self.integr.method())
        if self.io.restart:
            self.io.set_restart(self.grid, self.integr)
        else:
            _load_problem(problem, usr_dir)(self.grid, self.integr, usr_dir)
        # init_sim: ghost fill, cell B from the faces, cons (vanleer.pyx:41-53)
        self.ctx.set_state(self.grid.prim, self.grid.bfld)
        self.ctx.init()
        if self.io.restart:
            self.ctx.set_time(self.integr.time, self.integr.step)
        else:
            self.io.write_output(self)
        self.integr_params = {}
        self.coord_params = {}
        self._update_params()

    def _update_params(self):
        i = self.integr
        self.integr_params.update(time=i.time, step=i.step, dt=i.dt, tmax=i.tmax, cour=i.cour,
                                  char_proj=i.char_proj, gam=i.gam)
        gc = self.grid.coord
        self.coord_params.update(Nact=list(gc.Nact), Ntot=list(gc.Ntot), ng=gc.ng, lmin=list(gc.lmin),
                                 lmax=list(gc.lmax))

    def advance(self, tmax=None):
        """vanleer.advance: CFL steps until tmax (default: the config's tmax),
        writing output whenever the schedule says so."""
        tmax = self.integr.tmax if tmax is None else tmax
        while self.integr.time < tmax:
            self.ctx.advance(tmax, max_steps=1)
            t, s, dt = self.ctx.time()
            self.integr.time, self.integr.step, self.integr.dt = t, s, dt
            self.io.write_output(self)
            self.io.write_restart(self)
        self.io.flush()
        self._update_params()

    def _state(self):
        P, U, B = self.ctx.get_state()
        self.grid.prim[...] = P
        self.grid.cons[...] = U
        self.grid.bfld[...] = B

    @property
    def prim(self):
        self._state()
        return self.grid.prim

    @property
    def cons(self):
        self._state()
        return self.grid.cons

    @property
    def bfld(self):
        self._state()
        return self.grid.bfld
