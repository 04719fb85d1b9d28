"""Device parity of the plain (one kernel per reference loop) path.

exact_fp=True kernels are built without multiply-add contraction and must
reproduce the oracle bit for bit; the default kernels contract into DFMA and
must agree within 1e-12 relative per step (1e-9 after 100 steps)."""
import os

import numpy as np
import pytest

from helpers import device_ctx, oracle_sim, rel_err, setup_case

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("case", ["vortex", "blast", "turb3d", "cond3d"])
def test_golden_steps_bitwise(case):
    """From the golden initial state, the exact device path reproduces the
    steps the reference's compiled kernels produced (tests/golden/steps.npz)."""
    g = np.load(os.path.join(GOLD, "steps.npz"))
    n = int(g[case + "_n"][0])
    _, _, _, opts = setup_case(case, n=n)
    d = device_ctx(opts, exact_fp=True, path="plain")
    d.set_state(g[case + "_prim0"], g[case + "_bfld0"])
    d.init()
    for dt_ref in g[case + "_dts"]:
        assert d.new_dt() == dt_ref
        d.step(dt_ref)
    P, U, B = d.get_state()
    assert np.array_equal(P, g[case + "_prim"])
    assert np.array_equal(U, g[case + "_cons"])
    assert np.array_equal(B, g[case + "_bfld"])
    assert d.check() == 0


CASES = [("vortex", 32, {}), ("vortex", 32, dict(rsolver="hll")), ("vortex", 32, dict(rsolver="hllt")),
         ("vortex_pert", 32, dict(limiter="mc")), ("vortex_pert", 32, dict(limiter="mm")),
         ("vortex", 32, dict(reconstr="const")), ("blast", 32, {}), ("blast", 32, dict(outflow_face_aware=0)),
         ("turb3d", 12, {}), ("cond2d", 32, {}), ("cond2d", 32, dict(thcond_type="iso")),
         ("cond3d", 12, {}), ("cond3d", 12, dict(sat_hfe=1)), ("wave1d", 64, {}),
         ("vortex_pert", 32, dict(limiter="mc", charact_proj=1)), ("blast", 32, dict(charact_proj=1)),
         ("turb3d", 12, dict(charact_proj=1)), ("blast", 32, dict(grav=(0.3, -0.8, 0.0))),
         ("turb3d", 12, dict(grav=(0.0, 0.2, -0.4)))]


@pytest.mark.parametrize("case,n,kw", CASES)
def test_exact_mode_bitwise_vs_oracle(case, n, kw):
    kw = dict(kw)
    rc = kw.pop("reconstr", "linear")
    gc, prim, bfld, opts = setup_case(case, n=n, reconstr=rc)
    o = oracle_sim(opts, **kw)
    d = device_ctx(opts, exact_fp=True, path="plain", **kw)
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    for _ in range(4):
        dt = o.new_dt()
        assert d.new_dt() == dt
        o.step(dt)
        d.step(dt)
    for a, b in zip(o.get_state(), d.get_state()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case,n", [("vortex", 32), ("blast", 32), ("turb3d", 12), ("cond3d", 12)])
def test_fast_mode_per_step_tolerance(case, n):
    gc, prim, bfld, opts = setup_case(case, n=n)
    o = oracle_sim(opts)
    d = device_ctx(opts, path="plain")
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    for _ in range(3):
        # one step from identical states: relative difference per field <= 1e-12
        Po, _, Bo = o.get_state()
        d.set_state(Po, Bo)
        d.apply_bc()
        dt = o.new_dt()
        o.step(dt)
        d.step(dt)
        P1, U1, B1 = o.get_state()
        P2, U2, B2 = d.get_state()
        assert rel_err(P2, P1).max() <= 1e-12
        assert rel_err(B2, B1).max() <= 1e-12


def test_vortex_128_100_steps_fast():
    """Config-0 vortex 128^2, MC limiter: 100 steps within 1e-9 of the oracle."""
    gc, prim, bfld, opts = setup_case("vortex", n=128)
    o = oracle_sim(opts, limiter="mc")
    d = device_ctx(opts, limiter="mc", path="plain")
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    o.advance(10.0, max_steps=100)
    d.advance(10.0, max_steps=100)
    P1, _, B1 = o.get_state()
    P2, _, B2 = d.get_state()
    assert rel_err(P2, P1).max() <= 1e-9
    assert rel_err(B2, B1).max() <= 1e-9
    assert abs(d.time()[0] - o.time) <= 1e-12 * o.time


def test_nonphysical_state_is_reported():
    from bonzo_b200._lib import BnzError, BNZ_ERR_STATE
    gc, prim, bfld, opts = setup_case("vortex", n=16)
    d = device_ctx(opts, path="plain")
    prim[4][gc.active] = -1.0  # host-injected negative pressure
    d.set_state(prim, bfld)
    d.init()
    d.step(1e-3)
    with pytest.raises(BnzError) as e:
        d.check()
    assert e.value.code == BNZ_ERR_STATE
    assert d.check() == 0  # cleared by the read


@pytest.mark.parametrize("case,n", [("vortex_pert", 32), ("turb3d", 12)])
def test_driving_and_gravity_vs_oracle(case, n):
    """Turbulence driving (device sin/cos against libm: not bitwise) and gravity."""
    gc, prim, bfld, opts = setup_case(case, n=n)
    kw = dict(grav=(0.0, -0.4, 0.1), drive_f0=0.8, drive_tau=0.05, drive_nmod=1, drive_seed=11)
    o = oracle_sim(opts, **kw)
    d = device_ctx(opts, path="plain", **kw)
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    for _ in range(4):
        dt = o.new_dt()
        o.step(dt)
        d.step(dt)
    for a, b in zip(o.get_state(), d.get_state()):
        assert rel_err(a, b).max() <= 1e-12
