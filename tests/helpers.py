"""Shared test helpers: problem setup on both the oracle and the device."""
import numpy as np

from bonzo_b200 import problems as P

BC_NAMES = {"periodic": 0, "outflow": 1, "reflect": 2}


def setup_case(name, n=32, reconstr="linear", seed=0):
    """(GridCoord, prim, bfld, options) for a named small case."""
    if name == "vortex":
        gc = P.make_grid(n, n, 1, dims=2, bc=0, reconstr=reconstr)
        prim, bfld = P.otvortex(gc)
        opts = dict(dims=2, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4)
    elif name == "vortex_pert":
        gc = P.make_grid(n, n, 1, dims=2, bc=0, reconstr=reconstr)
        prim, bfld = P.otvortex(gc, pert_amp=1e-2, seed=seed)
        opts = dict(dims=2, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4)
    elif name == "blast":
        gc = P.make_grid(n, n, 1, dims=2, bc=1, reconstr=reconstr)
        prim, bfld = P.blast(gc, b_angle=0.7, center=(0.45, 0.55, 0.5), p_ratio=30.)
        opts = dict(dims=2, bc=((1, 1), (1, 1), (1, 1)), gam=5. / 3, cour=0.4)
    elif name == "blast_reflect":
        gc = P.make_grid(n, n, 1, dims=2, bc=2, reconstr=reconstr)
        prim, bfld = P.blast(gc, b_angle=0.3, center=(0.4, 0.6, 0.5), p_ratio=20.)
        prim[1][gc.active] = 0.3
        prim[2][gc.active] = -0.2
        opts = dict(dims=2, bc=((2, 2), (2, 2), (2, 2)), gam=5. / 3, cour=0.4)
    elif name == "mixed_bc":
        gc = P.make_grid(n, n, 1, dims=2, bc=((0, 0), (1, 1), (0, 0)), reconstr=reconstr)
        prim, bfld = P.otvortex(gc)
        opts = dict(dims=2, bc=((0, 0), (1, 1), (0, 0)), gam=5. / 3, cour=0.4)
    elif name == "turb3d":
        gc = P.make_grid(n, n, n, dims=3, bc=0, reconstr=reconstr)
        prim, bfld = P.turbulence3d(gc, seed=seed, kmax=min(16, n // 3))
        opts = dict(dims=3, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.3)
    elif name == "cond3d":
        gc = P.make_grid(n, n, n, dims=3, bc=0, reconstr=reconstr)
        prim, bfld = P.conduction3d(gc, seed=seed, kmax=min(8, n // 3))
        opts = dict(dims=3, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4, kappa0=0.01)
    elif name == "cond2d":
        gc = P.make_grid(n, n, 1, dims=2, bc=0, reconstr=reconstr)
        prim, bfld = P.thcond_gauss(gc)
        bfld[1][gc.active] = 0.05
        bfld[1][0, gc.j2 + 1, gc.i1:gc.i2 + 1] = 0.05
        opts = dict(dims=2, bc=((0, 0), (0, 0), (0, 0)), gam=2.0, cour=0.4, kappa0=0.02)
    elif name == "wave1d":
        gc = P.make_grid(n, 1, 1, dims=1, bc=0, reconstr=reconstr)
        prim, bfld, _ = P.linear_wave(gc, "fast", amp=1e-4)
        opts = dict(dims=1, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4)
    else:
        raise ValueError(name)
    opts.update(Nx=gc.Nact[0], Ny=gc.Nact[1], Nz=gc.Nact[2], reconstr=reconstr)
    return gc, prim, bfld, opts


def oracle_sim(opts, **kw):
    from oracle.oracle import OracleSim
    o = dict(opts)
    o.update(kw)
    return OracleSim(**o)


def device_ctx(opts, **kw):
    from bonzo_b200._lib import Context
    o = dict(opts)
    o.update(kw)
    return Context(**o)


def rel_err(a, b):
    """max |a - b| / max |b| per variable (0 where both vanish)."""
    out = []
    for x, y in zip(a, b):
        d = np.max(np.abs(x - y))
        s = np.max(np.abs(y))
        out.append(d / s if s > 0 else d)
    return np.array(out)


def active(arr, gc):
    k, j, i = gc.active
    return arr[:, k, j, i]
