"""Device parity of the split path (each face's flux formed once from per-cell
slopes in shared memory, cell EMFs formed on the fly, one fused update per
stage).

The exact build keeps the reference's arithmetic and must reproduce the oracle
bit for bit, ghost cells included, in 1D, 2D and 3D, for every Riemann solver,
limiter, boundary type and source term; sizes include tiles cut short at the
range ends.  The fast build must agree with the plain path and with the oracle
to the parity tolerance."""
import os

import numpy as np
import pytest

from bonzo_b200 import problems as P
from helpers import device_ctx, oracle_sim, rel_err, setup_case

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _run_pair(o, d, steps=4):
    for _ in range(steps):
        dt = o.new_dt()
        assert d.new_dt() == dt
        o.step(dt)
        d.step(dt)
    for a, b in zip(o.get_state(), d.get_state()):
        assert np.array_equal(a, b)


CASES = [("vortex", 32, {}), ("vortex", 32, dict(rsolver="hll")), ("vortex", 32, dict(rsolver="hllt")),
         ("vortex_pert", 32, dict(limiter="mc")), ("vortex_pert", 32, dict(limiter="mm")),
         ("vortex", 32, dict(reconstr="const")), ("blast", 33, {}), ("blast", 32, dict(outflow_face_aware=0)),
         ("blast_reflect", 29, {}), ("mixed_bc", 32, {}),
         ("turb3d", 12, {}), ("cond2d", 32, {}), ("cond3d", 12, dict(sat_hfe=1)),
         ("cond3d", 12, dict(thcond_type="iso")), ("cond3d", 14, dict(thcond_type="iso", sat_hfe=1)),
         ("wave1d", 64, {}),
         ("wave1d", 70, dict(reconstr="const")),
         ("vortex_pert", 32, dict(limiter="mc", charact_proj=1)), ("blast", 32, dict(charact_proj=1)),
         ("turb3d", 12, dict(charact_proj=1)), ("blast", 32, dict(grav=(0.3, -0.8, 0.0))),
         ("turb3d", 12, dict(grav=(0.0, 0.2, -0.4)))]


@pytest.mark.parametrize("case,n,kw", CASES)
def test_split_exact_bitwise_vs_oracle(case, n, kw):
    kw = dict(kw)
    rc = kw.pop("reconstr", "linear")
    gc, prim, bfld, opts = setup_case(case, n=n, reconstr=rc)
    o = oracle_sim(opts, **kw)
    d = device_ctx(opts, exact_fp=True, path="split", **kw)
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    _run_pair(o, d)
    assert d.check() == 0


def _case3(name, n, bc, reconstr="linear"):
    if name == "turb":
        gc = P.make_grid(*n, dims=3, bc=bc, reconstr=reconstr)
        prim, bfld = P.turbulence3d(gc, seed=0, kmax=min(6, min(n) // 3), mach=0.5)
    else:
        gc = P.make_grid(*n, dims=3, bc=bc, reconstr=reconstr)
        prim, bfld = P.blast(gc, b_mag=0.4, b_angle=0.6, center=(0.45, 0.55, 0.5), radius=0.2, p_ratio=40.)
        prim[3][gc.active] = 0.2
    bcs = bc if isinstance(bc, tuple) else ((bc, bc),) * 3
    return prim, bfld, dict(Nx=n[0], Ny=n[1], Nz=n[2], dims=3, bc=bcs, gam=5. / 3, cour=0.3, reconstr=reconstr)


CASES3 = [("turb", (24, 24, 24), 0, {}), ("turb", (32, 32, 32), 0, dict(limiter="mc")),
          ("blast", (24, 24, 24), 1, {}), ("blast", (32, 32, 32), 1, dict(rsolver="hll")),
          ("blast", (21, 19, 17), 1, {}), ("blast", (20, 22, 18), 2, dict(limiter="mm")),
          ("blast", (24, 20, 22), ((0, 0), (1, 1), (2, 2)), {}), ("turb", (20, 20, 20), 0, dict(charact_proj=1)),
          ("blast", (22, 22, 22), 2, dict(grav=(0.1, -0.3, 0.5))), ("turb", (40, 9, 70), 0, {}),
          ("blast", (16, 16, 16), 1, dict(reconstr="const"))]


@pytest.mark.parametrize("case,n,bc,kw", CASES3)
def test_split3d_exact_bitwise_vs_oracle(case, n, bc, kw):
    kw = dict(kw)
    prim, bfld, opts = _case3(case, n, bc, kw.pop("reconstr", "linear"))
    o = oracle_sim(opts, **kw)
    d = device_ctx(opts, exact_fp=True, path="split", **kw)
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    _run_pair(o, d)
    assert d.check() == 0


@pytest.mark.parametrize("case", ["vortex", "blast", "turb3d", "cond3d"])
def test_split_golden_steps_bitwise(case):
    """From the golden initial states made with the reference's compiled
    kernels (tests/golden/steps.npz), the split path reproduces their steps."""
    g = np.load(os.path.join(GOLD, "steps.npz"))
    n = int(g[case + "_n"][0])
    _, _, _, opts = setup_case(case, n=n)
    d = device_ctx(opts, exact_fp=True, path="split")
    d.set_state(g[case + "_prim0"], g[case + "_bfld0"])
    d.init()
    for dt_ref in g[case + "_dts"]:
        assert d.new_dt() == dt_ref
        d.step(dt_ref)
    P_, U, B = d.get_state()
    assert np.array_equal(P_, g[case + "_prim"])
    assert np.array_equal(U, g[case + "_cons"])
    assert np.array_equal(B, g[case + "_bfld"])


@pytest.mark.parametrize("case,n", [("vortex_pert", 32), ("turb3d", 12)])
def test_split_driving_equals_plain(case, n):
    """With the driving force (device sin/cos) and gravity on, the split and
    plain paths agree bit for bit in the exact build (and to the parity
    tolerance in the fast one)."""
    gc, prim, bfld, opts = setup_case(case, n=n)
    kw = dict(grav=(0.0, -0.4, 0.1), drive_f0=0.8, drive_tau=0.05, drive_nmod=1, drive_seed=11)
    for exact in (True, False):
        a = device_ctx(opts, path="plain", exact_fp=exact, **kw)
        b = device_ctx(opts, path="split", exact_fp=exact, **kw)
        for s in (a, b):
            s.set_state(prim, bfld)
            s.init()
        for _ in range(4):
            dt = a.new_dt()
            if exact:
                assert b.new_dt() == dt
            else:
                # the fast build contracts the paths' expressions differently
                assert abs(b.new_dt() - dt) <= 1e-13 * dt
            a.step(dt)
            b.step(dt)
        Pa, Ua, Ba = a.get_state()
        Pb, Ub, Bb = b.get_state()
        if exact:
            assert np.array_equal(Pa, Pb) and np.array_equal(Ua, Ub) and np.array_equal(Ba, Bb)
        else:
            assert rel_err(Pb, Pa).max() <= 1e-12
            assert rel_err(Bb, Ba).max() <= 1e-12


@pytest.mark.parametrize("steps", [1, 2, 5])
def test_split_graph_advance_matches_oracle_advance(steps):
    prim, bfld, opts = _case3("blast", (24, 24, 24), 1)
    o = oracle_sim(opts)
    d = device_ctx(opts, exact_fp=True, path="split")
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    o.advance(1e30, max_steps=steps)
    d.advance_graph(1e30, steps)
    t, nstep, _ = d.time()
    assert nstep == steps and t == o.time
    for a, b in zip(o.get_state(), d.get_state()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case,bc,kw", [("turb", 0, {}), ("turb", 0, dict(limiter="mc", charact_proj=1)),
                                        ("blast", 1, dict(rsolver="hll", limiter="mm"))])
def test_split3d_many_tiles_per_block_bitwise_vs_plain(case, bc, kw):
    """64^3: the corrector's flux sweeps run as persistent kernels that walk
    several tiles per block through two TMA-filled buffers in turn; in the
    exact build the state stays bitwise equal to the plain path's."""
    prim, bfld, opts = _case3(case, (64, 64, 64), bc)
    a = device_ctx(opts, exact_fp=True, path="plain", **kw)
    b = device_ctx(opts, exact_fp=True, path="split", **kw)
    for s in (a, b):
        s.set_state(prim, bfld)
        s.init()
    for _ in range(3):
        dt = a.new_dt()
        assert b.new_dt() == dt
        a.step(dt)
        b.step(dt)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    assert b.check() == 0


def test_split_fast_agrees_with_plain_3d():
    prim, bfld, opts = _case3("turb", (48, 48, 48), 0)
    a = device_ctx(opts, path="plain")
    b = device_ctx(opts, path="split")
    for s in (a, b):
        s.set_state(prim, bfld)
        s.init()
        s.advance_graph(1e30, 10)
    Pa, _, Ba = a.get_state()
    Pb, _, Bb = b.get_state()
    assert rel_err(Pb, Pa).max() <= 1e-11
    assert rel_err(Bb, Ba).max() <= 1e-11
    assert b.check() == 0


def test_split_vortex_128_100_steps_fast():
    """The vortex at 128^2 with the MC limiter: 100 steps within 1e-9 of the oracle."""
    gc, prim, bfld, opts = setup_case("vortex", n=128)
    o = oracle_sim(opts, limiter="mc")
    d = device_ctx(opts, limiter="mc", path="split")
    for s in (o, d):
        s.set_state(prim, bfld)
        s.init()
    o.advance(10.0, max_steps=100)
    d.advance(10.0, max_steps=100)
    P1, _, B1 = o.get_state()
    P2, _, B2 = d.get_state()
    assert rel_err(P2, P1).max() <= 1e-9
    assert rel_err(B2, B1).max() <= 1e-9


def test_split_nonphysical_state_is_reported():
    from bonzo_b200._lib import BnzError, BNZ_ERR_STATE
    gc, prim, bfld, opts = setup_case("vortex", n=16)
    d = device_ctx(opts, path="split")
    prim[4][gc.active] = -1.0
    d.set_state(prim, bfld)
    d.init()
    d.step(1e-3)
    with pytest.raises(BnzError) as e:
        d.check()
    assert e.value.code == BNZ_ERR_STATE
    assert d.check() == 0


@pytest.mark.parametrize("path", ["split", "plain", "fused"])
@pytest.mark.parametrize("case,n", [("vortex", 32), ("turb3d", 12)])
def test_fixed_dt_advance_matches_oracle(path, case, n):
    """fixdt (vanleer.pyx:87-99): every step takes dt_fixed, with no clip to
    tmax; the loop stops once the time has reached tmax.  The host loop on
    every path, and graph stepping past tmax on the split and fused paths
    (further steps take dt = 0 and leave the state as it is)."""
    gc, prim, bfld, opts = setup_case(case, n=n)
    kw = dict(fixdt=True, dt_fixed=1.25e-3)
    tmax = 0.0106  # not a multiple of dt_fixed: the last step overshoots
    o = oracle_sim(opts, **kw)
    o.set_state(prim, bfld)
    o.init()
    o.advance(tmax)
    runs = [("host", None)] + ([("graph", 14)] if path != "plain" else [])
    for how, nsteps in runs:
        d = device_ctx(opts, exact_fp=True, path=path, **kw)
        d.set_state(prim, bfld)
        d.init()
        if how == "host":
            d.advance(tmax)
        else:
            d.advance_graph(tmax, nsteps)
        t, s, _ = d.time()
        assert t == o.time and s == o.nstep, (how, t, o.time, s, o.nstep)
        for a, b in zip(o.get_state(), d.get_state()):
            assert np.array_equal(a, b), how
