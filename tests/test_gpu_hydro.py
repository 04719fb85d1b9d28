"""The hydro build (MFIELD 0) on the device: HLLC and the hydro HLL.

The reference compiles HLLC only without a magnetic field (fluxes_c.c:230-327
under #if !MFIELD).  The device's hydro mode holds the field at zero, skips
constrained transport on the plain path (the split path runs it on zero
fields) and uses the hydro sound speed; its kernels must equal
the reference's hydro-build kernels (tests/golden/kernels_hydro.npz, made by
the reference's own compiled code) bit for bit in the exact build, and its
steps the oracle's hydro build.  The device Riemann entry point (the
reference's C-level flux call, bnz_riemann) is pinned against the MHD
fixtures too.
"""
import os

import numpy as np
import pytest

from bonzo_b200 import problems as P
from helpers import device_ctx, oracle_sim, rel_err

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _flux(rs, g, key, exact):
    import torch
    from bonzo_b200._lib import riemann
    wl = torch.from_numpy(g[key + "_wl"]).cuda()
    wr = torch.from_numpy(g[key + "_wr"]).cuda()
    bx = torch.from_numpy(g[key + "_bx"]).cuda()
    return riemann(rs, wl, wr, bx, float(g["gam"]), exact_fp=exact).cpu().numpy()


@pytest.mark.parametrize("rs", ["hll", "hllc"])
def test_hydro_riemann_vs_reference_kernels(rs):
    g = np.load(os.path.join(GOLD, "kernels_hydro.npz"))
    f = _flux(rs, g, rs, exact=True)
    assert np.array_equal(f, g[rs + "_flux"])
    f = _flux(rs, g, rs, exact=False)
    assert rel_err(f, g[rs + "_flux"]).max() <= 1e-13


@pytest.mark.parametrize("rs", ["hll", "hllt", "hlld"])
def test_mhd_riemann_vs_reference_kernels(rs):
    """The same entry point on the MHD fixtures (every HLLD fan region, Bx = 0)."""
    g = np.load(os.path.join(GOLD, "kernels_mhd.npz"))
    f = _flux(rs, g, rs, exact=True)
    assert np.array_equal(f, g[rs + "_flux"])


def _hydro_case(n, dims=2, bc=1, seed=0):
    rng = np.random.default_rng(seed)
    nz = n if dims == 3 else 1
    gc = P.make_grid(n, n, nz, dims=dims, bc=bc)
    prim, bfld = P.blast(gc, b_mag=0.0, center=(rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7), 0.5),
                         p_ratio=rng.uniform(10, 100))
    a = gc.active
    prim[1][a] = 0.2  # a uniform stream through the box
    prim[5][a] = np.where(prim[4][a] > 0.5, 1.0, 0.0)  # passive scalar marks the blast
    bcs = tuple((bc, bc) for _ in range(3))
    opts = dict(Nx=n, Ny=n, Nz=nz, dims=dims, bc=bcs, gam=1.4, cour=0.4)
    return gc, prim, bfld, opts


@pytest.mark.parametrize("path", ["plain", "split"])
@pytest.mark.parametrize("rs,limiter,dims,bc", [("hllc", "vl", 2, 1), ("hllc", "mc", 2, 0), ("hll", "vl", 2, 1),
                                                 ("hllc", "mm", 3, 0), ("hll", "mc", 3, 1), ("hllc", "vl", 2, 2)])
def test_hydro_step_bitwise_vs_oracle(rs, limiter, dims, bc, path):
    n = 40 if dims == 2 else 14
    gc, prim, bfld, opts = _hydro_case(n, dims, bc)
    o = oracle_sim(opts, rsolver=rs, limiter=limiter, hydro=True)
    d = device_ctx(opts, rsolver=rs, limiter=limiter, hydro=True, exact_fp=True, path=path)
    o.set_state(prim[:6], bfld)
    d.set_state(prim, bfld)
    o.init()
    d.init()
    for _ in range(5):
        dt = o.new_dt()
        assert d.new_dt() == dt
        o.step(dt)
        d.step(dt)
    Po, Uo, _ = o.get_state()
    Pd, Ud, Bd = d.get_state()
    assert np.array_equal(Pd[:6], Po)
    assert np.array_equal(Ud[:6], Uo)
    assert not Pd[6:].any() and not Bd.any()
    assert d.check() == 0


@pytest.mark.parametrize("path", ["plain", "split"])
def test_hydro_fast_100_steps_vs_oracle(path):
    gc, prim, bfld, opts = _hydro_case(96, 2, 1, seed=3)
    o = oracle_sim(opts, rsolver="hllc", hydro=True)
    d = device_ctx(opts, rsolver="hllc", hydro=True, path=path)
    o.set_state(prim[:6], bfld)
    d.set_state(prim, bfld)
    o.init()
    d.init()
    o.advance(1e30, max_steps=100)
    d.advance_graph(1e30, 100)
    assert abs(d.time()[0] - o.time) <= 1e-12 * o.time
    Po, _, _ = o.get_state()
    Pd, _, _ = d.get_state()
    assert rel_err(Pd[:6], Po).max() <= 1e-9
    assert d.check() == 0


def test_hydro_split_batch3d_bitwise_vs_oracle():
    """A 3D batch of the hydro build on the split path, each instance with its
    own CFL dt, against each grid alone in the oracle's hydro build."""
    from bonzo_b200._lib import Batch
    inst = [_hydro_case(14, 3, 0, seed=1), _hydro_case(12, 3, 1, seed=2)]
    b = Batch([dict(Nx=o["Nx"], Ny=o["Ny"], Nz=o["Nz"], dims=3, bc=o["bc"]) for _, _, _, o in inst],
              gam=1.4, cour=0.4, rsolver="hllc", hydro=True, exact_fp=True, path="split")
    for q, (gc, prim, bfld, opts) in enumerate(inst):
        b[q].set_state(prim, bfld)
        b[q].init()
    b.advance(1e30, 3)
    for q, (gc, prim, bfld, opts) in enumerate(inst):
        o = oracle_sim(opts, rsolver="hllc", hydro=True)
        o.set_state(prim[:6], bfld)
        o.init()
        o.advance(1e30, max_steps=3)
        assert b[q].time()[1] == 3 and b[q].time()[0] == o.time
        Po, Uo, _ = o.get_state()
        Pd, Ud, Bd = b[q].get_state()
        assert np.array_equal(Pd[:6], Po) and np.array_equal(Ud[:6], Uo)
        assert not Bd.any()
