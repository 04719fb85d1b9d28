"""config.cfg writers for the Simulation facade tests."""
import os

VORTEX_CFG = """[computation]
Nx: {n}
Ny: {n}
Nz: 1
Lx: 1.
Ly: 1.
Lz: 1.
tmax: {tmax}
cour: 0.4
cour_diff: 0.5
rsolver: hlld
reconstr: linear
limiter: mc
charact_proj: 0

[physics]
bc_x1: 0
bc_x2: 0
bc_y1: 0
bc_y2: 0
bc_z1: 0
bc_z2: 0
gam: 1.6666666666666667
kappa0: 0
elec_thcond_type: aniso
sat_hfe: 0

[problem]
name: otvortex
pert_amp: 0.01
seed: 2

[output]
hst_dt: {hst_dt}
grid_dt: {grid_dt}
slc_dt: 0.
slc_axis: z
slc_pos_ind: 0
var_type: prim
write_ghost: {ghost}

[restart]
restart: {restart}
rst_dt: {rst_dt}
"""


def write_cfg(usr_dir, n=32, tmax=0.02, hst_dt=0.005, grid_dt=0.01, ghost=0, restart=0, rst_dt=0.0):
    os.makedirs(usr_dir, exist_ok=True)
    with open(os.path.join(usr_dir, "config.cfg"), "w") as f:
        f.write(VORTEX_CFG.format(n=n, tmax=tmax, hst_dt=hst_dt, grid_dt=grid_dt, ghost=ghost, restart=restart,
                                  rst_dt=rst_dt))


def write_cfg3d(usr_dir, n=16, tmax=0.01, kappa0=0.0):
    """A 3D decaying-turbulence run (the facade runs it on the split path)."""
    os.makedirs(usr_dir, exist_ok=True)
    cfg = VORTEX_CFG.format(n=n, tmax=tmax, hst_dt=0., grid_dt=0., ghost=0, restart=0, rst_dt=0.)
    cfg = cfg.replace("Nz: 1\n", "Nz: %d\n" % n).replace("cour: 0.4", "cour: 0.3").replace("limiter: mc", "limiter: vl")
    cfg = cfg.replace("kappa0: 0\n", "kappa0: %r\n" % kappa0)
    cfg = cfg.replace("name: otvortex\npert_amp: 0.01\nseed: 2\n", "name: turbulence3d\nseed: 3\nmach: 0.5\nkmax: 4\n")
    with open(os.path.join(usr_dir, "config.cfg"), "w") as f:
        f.write(cfg)
