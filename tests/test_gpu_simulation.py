"""The Simulation facade on the device: a run from config.cfg against the
oracle, the history file against host sums, grid output files, restart
continuation, and the asynchronous snapshot."""
import glob
import os

import numpy as np
import pytest

from sim_cases import write_cfg, write_cfg3d

pytestmark = pytest.mark.gpu


def test_simulation_matches_oracle_and_writes_output(tmp_path):
    from bonzo_b200 import problems
    from bonzo_b200.simulation import CONS_NAMES, PRIM_NAMES, B_NAMES, Simulation
    from oracle.oracle import OracleSim
    d = str(tmp_path)
    write_cfg(d, n=32, tmax=0.02, hst_dt=0.005, grid_dt=0.01)
    sim = Simulation(d)
    # the same problem on the oracle
    prim, bfld = problems.otvortex(sim.grid.coord, pert_amp=0.01, seed=2)
    o = OracleSim(Nx=32, Ny=32, Nz=1, dims=2, bc=sim.grid.bc, gam=5. / 3, cour=0.4, rsolver="hlld", limiter="mc")
    o.set_state(prim, bfld)
    o.init()
    sim.advance()
    o.advance(0.02)
    P, U, B = o.get_state()
    assert sim.integr.step == o.nstep and abs(sim.integr.time - 0.02) < 1e-15
    for a, b in ((sim.prim, P), (sim.bfld, B)):
        for v in range(a.shape[0]):
            assert np.abs(a[v] - b[v]).max() <= 1e-11 * max(np.abs(b[v]).max(), 1e-300)
    # history: header + rows at t = 0, 0.005, ..., 0.02
    rows = np.loadtxt(os.path.join(d, "out", "hst.txt"), skiprows=1)
    assert rows.shape == (5, 16)
    u = sim.cons[:, 0, 3:35, 3:35]
    ek = 0.5 / u[0] * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2)
    em = 0.5 * (u[6] ** 2 + u[7] ** 2 + u[8] ** 2)
    ref = [u[0].mean(), ek.mean(), (u[4] - ek - em).mean(), em.mean(), u[4].mean(), u[1].mean(), u[2].mean(),
           u[3].mean(), u[6].mean(), u[7].mean(), u[8].mean()]
    ref += [np.sqrt(abs((u[6 + q] ** 2).mean() - u[6 + q].mean() ** 2)) for q in range(3)]
    last = rows[-1]
    assert last[0] == sim.integr.step and abs(last[1] - 0.02) < 1e-12
    assert np.allclose(last[2:], ref, rtol=1e-6, atol=1e-12)   # the file keeps 7 digits ('{:<14e}')
    assert np.allclose(sim.ctx.history()[2:], ref, rtol=1e-13, atol=1e-15)
    # full-grid files at t = 0, 0.01, 0.02 with the reference's dataset names
    files = sorted(glob.glob(os.path.join(d, "out", "grid_*.npz")))
    assert [os.path.basename(f) for f in files] == ["grid_000.npz", "grid_001.npz", "grid_002.npz"]
    with np.load(files[-1]) as f:
        for n, name in enumerate(PRIM_NAMES + B_NAMES[:3]):
            assert np.array_equal(f[name], sim.prim[n, :, 3:35, 3:35])
        for n in range(3):
            assert np.array_equal(f[B_NAMES[3 + n]], sim.bfld[n, :, 3:35, 3:35])
        assert float(f["time"]) == sim.integr.time and int(f["step"]) == sim.integr.step
        assert f["xf"].shape == (39,)
    assert CONS_NAMES[1] == "mx"


def test_restart_continues_bitwise(tmp_path):
    from bonzo_b200.simulation import Simulation
    a = str(tmp_path / "a")
    write_cfg(a, n=24, tmax=0.01, hst_dt=0.0, grid_dt=0.0, rst_dt=0.01)
    s1 = Simulation(a)
    s1.advance(0.01)
    assert os.path.exists(os.path.join(a, "rst", "rst_grid.npz"))
    # restart from the file and continue to 0.02
    write_cfg(a, n=24, tmax=0.02, hst_dt=0.0, grid_dt=0.0, rst_dt=0.0, restart=1)
    s2 = Simulation(a)
    assert s2.integr.time == 0.01 and s2.integr.step == s1.integr.step
    s2.advance(0.02)
    # the same run without the restart
    c = str(tmp_path / "c")
    write_cfg(c, n=24, tmax=0.02, hst_dt=0.0, grid_dt=0.0)
    s3 = Simulation(c)
    s3.advance(0.01)
    s3.advance(0.02)
    assert s2.integr.step == s3.integr.step
    assert np.array_equal(s2.prim, s3.prim)
    assert np.array_equal(s2.bfld, s3.bfld)


def test_snapshot_equals_state(tmp_path):
    from bonzo_b200.simulation import Simulation
    d = str(tmp_path)
    write_cfg(d, n=24, tmax=0.005, hst_dt=0.0, grid_dt=0.0)
    s = Simulation(d)
    s.advance()
    P = np.empty((9,) + s.ctx.shape)
    U = np.empty((9,) + s.ctx.shape)
    B = np.empty((3,) + s.ctx.shape)
    s.ctx.snapshot(P, U, B)
    s.ctx.snapshot_wait()
    P2, U2, B2 = s.ctx.get_state()
    assert np.array_equal(P, P2) and np.array_equal(U, U2) and np.array_equal(B, B2)


@pytest.mark.parametrize("kappa0", [0.0, 0.01])
def test_simulation_3d_runs_on_split_path(tmp_path, kappa0):
    """A 3D run from config.cfg goes through the split path and matches the
    oracle (the facade's fast build: 1e-11 relative), conduction included."""
    from bonzo_b200 import problems
    from bonzo_b200._lib import PATH
    from bonzo_b200.simulation import Simulation
    from oracle.oracle import OracleSim
    d = str(tmp_path)
    write_cfg3d(d, n=16, tmax=0.01, kappa0=kappa0)
    sim = Simulation(d)
    assert sim.ctx.method_desc.path == PATH["split"]
    prim, bfld = problems.turbulence3d(sim.grid.coord, seed=3, mach=0.5, kmax=4)
    o = OracleSim(Nx=16, Ny=16, Nz=16, dims=3, bc=sim.grid.bc, gam=5. / 3, cour=0.3, rsolver="hlld", limiter="vl",
                  kappa0=kappa0)
    o.set_state(prim, bfld)
    o.init()
    sim.advance()
    o.advance(0.01)
    P, U, B = o.get_state()
    assert sim.integr.step == o.nstep and abs(sim.integr.time - 0.01) < 1e-15
    for a, b in ((sim.prim, P), (sim.cons, U), (sim.bfld, B)):
        for v in range(a.shape[0]):
            assert np.abs(a[v] - b[v]).max() <= 1e-11 * max(np.abs(b[v]).max(), 1e-300)
