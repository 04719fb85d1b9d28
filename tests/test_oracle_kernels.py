"""Pin the oracle's restated kernels to the reference's own compiled kernels.

Golden vectors in tests/golden/ were produced by the reference's C kernels
(src/mhd/fluxes_c.c, src/mhd/eos_c.{c,h}, src/coordinates/reconstr_c.c built
by oracle/build_ref.py) -- see tests/golden/make_golden.py.  Every comparison
here is bitwise.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
EN = 4


@pytest.fixture(scope="module")
def gm():
    return np.load(os.path.join(GOLD, "kernels_mhd.npz"))


@pytest.fixture(scope="module")
def gh():
    return np.load(os.path.join(GOLD, "kernels_hydro.npz"))


@pytest.mark.parametrize("rs", ["hll", "hlld"])
def test_riemann_mhd_bitwise(gm, rs):
    f = O.orc_flux_flat(rs, gm[rs + "_wl"], gm[rs + "_wr"], gm[rs + "_bx"], float(gm["gam"]))
    assert np.array_equal(f, gm[rs + "_flux"])


def test_hllt_bitwise_except_energy(gm):
    # fluxes_c.c:447-607 reads its star-state energy entries uninitialised
    # (undefined behaviour); every other component must match exactly.
    f = O.orc_flux_flat("hllt", gm["hllt_wl"], gm["hllt_wr"], gm["hllt_bx"], float(gm["gam"]))
    ref = gm["hllt_flux"]
    keep = [n for n in range(9) if n != EN]
    assert np.array_equal(f[keep], ref[keep])


def test_hlld_covers_degenerate_and_supersonic(gm):
    bx = gm["hlld_bx"]
    assert (bx == 0).sum() > 10
    vx = gm["hlld_wl"][1]
    assert (vx == 8.0).sum() > 10 and (vx == -8.0).sum() > 10


def test_eos_bitwise(gm):
    g = float(gm["gam"])
    assert np.array_equal(O.orc_row_eos("prim2cons_1", gm["eos_w"], g), gm["eos_u"])
    assert np.array_equal(O.orc_row_eos("cons2prim_1", gm["eos_u"], g), gm["eos_w_back"])
    w = gm["eos_w"]
    cf = np.array([O.orc_fms(w[:, q], g) for q in range(w.shape[1])])
    assert np.array_equal(cf, gm["fms"])


@pytest.mark.parametrize("fn,order,cp", [("reconstr_const", 0, 0), ("reconstr_linear", 1, 0),
                                         ("reconstr_linear", 1, 1)])
def test_reconstruction_bitwise(gm, fn, order, cp):
    wl, wr = O.reconstr_with(fn, order, gm["rc_w"], float(gm["gam"]), char_proj=cp)
    n = gm["rc_w"].shape[1]
    # the reference writes wr[1..n-2] and wl[2..n-1]
    assert np.array_equal(wr[:, 1:n - 1], gm["rc_%s_cp%d_wr" % (fn, cp)][:, 1:n - 1])
    assert np.array_equal(wl[:, 2:n], gm["rc_%s_cp%d_wl" % (fn, cp)][:, 2:n])


@pytest.mark.parametrize("rs", ["hll", "hllc", "hllt"])
def test_riemann_hydro_bitwise(gh, rs):
    f = O.orc_flux_flat(rs, gh[rs + "_wl"], gh[rs + "_wr"], gh[rs + "_bx"], float(gh["gam"]), hydro=True)
    assert np.array_equal(f, gh[rs + "_flux"])


def test_reconstruction_hydro_bitwise(gh):
    wl, wr = O.reconstr_with("reconstr_linear", 1, gh["rc_w"], float(gh["gam"]), hydro=True)
    n = gh["rc_w"].shape[1]
    assert np.array_equal(wr[:, 1:n - 1], gh["rc_wr"][:, 1:n - 1])
    assert np.array_equal(wl[:, 2:n], gh["rc_wl"][:, 2:n])


@pytest.mark.parametrize("case", ["vortex", "blast", "turb3d", "cond3d"])
def test_oracle_steps_match_reference_kernels(case):
    """Whole VL2 steps with the restated kernels equal the same steps run on
    the reference's compiled kernels (golden)."""
    from helpers import setup_case
    g = np.load(os.path.join(GOLD, "steps.npz"))
    n = int(g[case + "_n"][0])
    gc, _, _, opts = setup_case(case, n=n)
    sim = O.OracleSim(**opts)
    sim.set_state(g[case + "_prim0"], g[case + "_bfld0"])
    sim.init()
    for dt_ref in g[case + "_dts"]:
        dt = sim.new_dt()
        assert dt == dt_ref
        sim.step(dt)
    P, U, B = sim.get_state()
    assert np.array_equal(P, g[case + "_prim"])
    assert np.array_equal(U, g[case + "_cons"])
    assert np.array_equal(B, g[case + "_bfld"])


needs_ref = pytest.mark.skipif(O.ref_lib() is None, reason="reference kernels (oracle/_ref) not built")


@needs_ref
@pytest.mark.parametrize("rs", ["hll", "hlld"])
def test_live_random_vs_reference(rs):
    rng = np.random.default_rng(7)
    n = 5000
    wl = np.abs(rng.normal(1, 0.5, (9, n))) + 0.05
    wr = np.abs(rng.normal(1, 0.5, (9, n))) + 0.05
    wl[1:4] = rng.normal(0, 2, (3, n))
    wr[1:4] = rng.normal(0, 2, (3, n))
    wl[6:9] = rng.normal(0, 1, (3, n))
    wr[6:9] = rng.normal(0, 1, (3, n))
    bx = rng.normal(0, 1, n)
    assert np.array_equal(O.orc_flux_flat(rs, wl, wr, bx, 1.4), O.ref_flux_flat(rs, wl, wr, bx, 1.4))


@needs_ref
def test_live_steps_with_reference_kernels():
    from helpers import setup_case, oracle_sim
    gc, prim, bfld, opts = setup_case("vortex_pert", n=24)
    a = oracle_sim(opts)
    b = oracle_sim(opts, use_ref_kernels=True)
    for s in (a, b):
        s.set_state(prim, bfld)
        s.init()
        s.advance(1.0, max_steps=4)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
