"""Host side of the Simulation facade: config -> grid / integrator / I/O,
output schedule, history file header, problem loading (no GPU needed)."""
import os

import numpy as np
import pytest

from sim_cases import write_cfg


def test_grid_and_integrator_from_config(tmp_path):
    from bonzo_b200.simulation import BnzGrid, BnzIntegr
    write_cfg(str(tmp_path), n=24)
    g = BnzGrid(str(tmp_path))
    i = BnzIntegr(g.coord, str(tmp_path))
    assert g.dims == 2 and g.coord.Nact[:2] == [24, 24] and g.coord.ng == 3
    assert g.prim.shape == (9, 1, 30, 30) and g.bfld.shape == (3, 1, 30, 30)
    assert i.rsolver == "hlld" and i.limiter == "mc" and abs(i.gam - 5. / 3) < 1e-15
    assert i.tmax == 0.02 and i.time == 0.0 and i.step == 0
    assert i.grav == (0.0, 0.0, 0.0) and i.drive_f0 == 0.0 and i.drive_nmod == 1


def test_io_header_and_schedule(tmp_path):
    from bonzo_b200.simulation import HST_NAMES, BnzIO
    write_cfg(str(tmp_path), hst_dt=0.005)
    io = BnzIO(str(tmp_path))
    head = open(os.path.join(str(tmp_path), "out", "hst.txt")).read()
    assert head.split() == HST_NAMES
    assert os.path.isdir(os.path.join(str(tmp_path), "rst"))
    # io.pyx:137-140: due when the step crossed a multiple of the interval
    assert BnzIO._due(0.0051, 0.0002, 0.005)
    assert not BnzIO._due(0.0056, 0.0002, 0.005)
    assert BnzIO._due(0.0, 1e-6, 0.005)       # initial output
    assert not BnzIO._due(0.3, 0.1, 0.0)      # switched off


def test_problem_loading(tmp_path):
    from bonzo_b200 import problems
    from bonzo_b200.config import ConfigError
    from bonzo_b200.simulation import BnzGrid, BnzIntegr, _load_problem
    write_cfg(str(tmp_path), n=16)
    g = BnzGrid(str(tmp_path))
    i = BnzIntegr(g.coord, str(tmp_path))
    f = _load_problem(None, str(tmp_path))       # [problem] name: otvortex
    assert f is problems.SET_PROBLEM["otvortex"]
    f(g, i, str(tmp_path))
    a = g.coord.active
    assert np.allclose(g.prim[0][a], (5. / 3) ** 2) and np.allclose(g.prim[4][a], 5. / 3)
    # faces from a vector potential: discrete divergence vanishes
    gc = g.coord
    bx, by = g.bfld[0, 0], g.bfld[1, 0]
    dx, dy = gc.dlf[0][gc.i1], gc.dlf[1][gc.j1]
    div = ((bx[gc.j1:gc.j2 + 1, gc.i1 + 1:gc.i2 + 2] - bx[gc.j1:gc.j2 + 1, gc.i1:gc.i2 + 1]) / dx +
           (by[gc.j1 + 1:gc.j2 + 2, gc.i1:gc.i2 + 1] - by[gc.j1:gc.j2 + 1, gc.i1:gc.i2 + 1]) / dy)
    assert np.abs(div).max() < 1e-10
    # a user problem.py in usr_dir
    d2 = tmp_path / "user"
    write_cfg(str(d2), n=16)
    cfgtxt = open(d2 / "config.cfg").read().replace("name: otvortex", "")
    open(d2 / "config.cfg", "w").write(cfgtxt)
    (d2 / "problem.py").write_text("def set_problem(grid, integr, usr_dir):\n    grid.prim[0] = 7.0\n")
    f = _load_problem(None, str(d2))
    f(g, i, str(d2))
    assert np.all(g.prim[0] == 7.0)
    with pytest.raises(ConfigError):
        _load_problem("no_such_problem", str(tmp_path))
