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
