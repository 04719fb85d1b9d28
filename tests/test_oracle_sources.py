"""Source terms of the oracle's step (test infrastructure pinned by physics):
constant gravity on a uniform periodic box, and the turbulence driving force
(zero net momentum input, reproducible from its seed)."""
import numpy as np
import pytest

from helpers import oracle_sim


def _uniform(n, dims=2):
    from bonzo_b200 import problems as P
    gc = P.make_grid(n, n if dims >= 2 else 1, n if dims >= 3 else 1, dims=dims, bc=0)
    prim, bfld = P._empty(gc)
    a = gc.active
    prim[0][a] = 1.3
    prim[4][a] = 0.7
    bfld[0][...] = 0.3
    bfld[1][...] = 0.2
    opts = dict(Nx=gc.Nact[0], Ny=gc.Nact[1], Nz=gc.Nact[2], dims=dims, bc=((0, 0), (0, 0), (0, 0)),
                gam=5. / 3, cour=0.4)
    return gc, prim, bfld, opts


def test_gravity_on_a_uniform_box_is_exact_kinematics():
    gc, prim, bfld, opts = _uniform(16)
    g = (0.2, -0.5, 0.0)
    o = oracle_sim(opts, grav=g)
    o.set_state(prim, bfld)
    o.init()
    t = 0.0
    for dt in (0.01, 0.02, 0.015):
        o.step(dt)
        t += dt
    P, U, B = o.get_state()
    a = gc.active
    rho = 1.3
    assert np.allclose(P[1][a], g[0] * t, rtol=1e-12, atol=1e-14)
    assert np.allclose(P[2][a], g[1] * t, rtol=1e-12, atol=1e-14)
    assert np.allclose(P[0][a], rho, rtol=1e-14)
    # the midpoint rule is exact for the linear velocity: E_kin = rho g^2 t^2 / 2
    # and the pressure does not change
    assert np.allclose(P[4][a], 0.7, rtol=1e-12)
    ek = 0.5 * rho * (P[1][a] ** 2 + P[2][a] ** 2)
    assert np.allclose(ek, 0.5 * rho * (g[0] ** 2 + g[1] ** 2) * t * t, rtol=1e-11)


@pytest.mark.parametrize("dims", [2, 3])
def test_driving_adds_no_net_momentum_and_is_seeded(dims):
    n = 16 if dims == 2 else 8
    gc, prim, bfld, opts = _uniform(n, dims)
    runs = []
    for seed in (5, 5, 6):
        o = oracle_sim(opts, drive_f0=0.5, drive_tau=0.1, drive_nmod=1, drive_seed=seed)
        o.set_state(prim, bfld)
        o.init()
        for _ in range(3):
            o.step(0.005)
        runs.append(o.get_state())
    a = gc.active
    P = runs[0][0]
    # driven velocity appears; the force has no k = 0 mode, so the mean momentum stays zero
    assert np.abs(P[1][a]).max() > 1e-4
    U = runs[0][1]
    for n_ in (1, 2, 3):
        assert abs(U[n_][a].mean()) < 1e-14 * max(np.abs(U[n_][a]).max(), 1.0)
    assert np.array_equal(runs[0][0], runs[1][0])
    assert not np.array_equal(runs[0][0], runs[2][0])
