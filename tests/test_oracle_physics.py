"""Invariants and known answers of the oracle's step (the checker itself).

The reference ships no tests; these pin the restated orchestration with
properties the method guarantees: constrained transport keeps the face
divergence at round-off, the conservative update conserves mass / momentum /
energy on periodic grids, RKL2 conduction reproduces the analytic Gaussian
(scripts/thcond1d.py) and the scheme converges at second order on a linear
MHD wave.
"""
import math

import numpy as np
import pytest

from bonzo_b200 import problems as P
from helpers import oracle_sim, setup_case


def div_b(gc, B, prim):
    ks, js, is_ = gc.active
    dx = gc.dlf[0][gc.i1]
    d = (B[0][ks, js, gc.i1 + 1:gc.i2 + 2] - B[0][ks, js, is_]) / dx
    if gc.dims >= 2:
        d = d + (B[1][ks, gc.j1 + 1:gc.j2 + 2, is_] - B[1][ks, js, is_]) / gc.dlf[1][gc.j1]
    if gc.dims >= 3:
        d = d + (B[2][gc.k1 + 1:gc.k2 + 2, js, is_] - B[2][ks, js, is_]) / gc.dlf[2][gc.k1]
    bmag = np.sqrt((prim[6:9][:, ks, js, is_] ** 2).sum(0)).max()
    return np.abs(d).max() * dx / bmag


@pytest.mark.parametrize("case,n,steps", [("vortex", 32, 10), ("blast", 24, 10), ("turb3d", 10, 5),
                                          ("cond3d", 10, 4), ("vortex_pert", 32, 10)])
def test_divb_roundoff(case, n, steps):
    gc, prim, bfld, opts = setup_case(case, n=n)
    s = oracle_sim(opts)
    s.set_state(prim, bfld)
    s.init()
    P0, _, B0 = s.get_state()
    assert div_b(gc, B0, P0) <= 1e-13
    s.advance(10.0, max_steps=steps)
    P1, _, B1 = s.get_state()
    assert div_b(gc, B1, P1) <= 1e-13


@pytest.mark.parametrize("case,n", [("vortex", 32), ("turb3d", 10), ("cond3d", 10)])
def test_conservation_periodic(case, n):
    gc, prim, bfld, opts = setup_case(case, n=n)
    s = oracle_sim(opts)
    s.set_state(prim, bfld)
    s.init()
    _, U0, _ = s.get_state()
    s.advance(10.0, max_steps=6)
    _, U1, _ = s.get_state()
    a = gc.active
    for v in (0, 4):  # mass, total energy
        s0, s1 = U0[v][a].sum(), U1[v][a].sum()
        assert abs(s1 - s0) <= 1e-13 * abs(s0) * 10
    for v in (1, 2, 3):  # momentum (scale by total mass x max speed)
        scale = U0[0][a].sum() * (np.abs(U0[v][a] / U0[0][a]).max() + 1)
        assert abs(U1[v][a].sum() - U0[v][a].sum()) <= 1e-12 * scale


@pytest.mark.parametrize("aniso", ["aniso", "iso"])
def test_gaussian_diffusion_known_answer(aniso):
    """thcond_gauss.pyx IC, diffusion only, vs g(x,t) of scripts/thcond1d.py
    with a = (gamma-1) kappa0 = 0.02, sigma = 0.15, L = 2."""
    N, L, sig, kappa0, gam = 200, 2.0, 0.15, 0.02, 2.0
    gc = P.make_grid(N, 1, 1, dims=1, bc=0, lmax=(L, 1., 1.))
    prim, bfld = P.thcond_gauss(gc, sig=sig, bx=0.1)
    s = oracle_sim(dict(Nx=N, Ny=1, Nz=1, dims=1, lmax=(L, 1., 1.), gam=gam, kappa0=kappa0,
                        thcond_type=aniso, cour_diff=0.5))
    s.set_state(prim, bfld)
    s.init()
    t, dt = 0.0, 0.002
    while t < 0.3 - 1e-12:
        s.L.orc_diffuse(s.h, dt)
        t += dt
    Pn, _, _ = s.get_state()
    a = (gam - 1) * kappa0
    x = gc.lv[0][gc.i1:gc.i2 + 1]
    g = 1. / math.sqrt(1 + 4 * a * t / sig ** 2) * np.exp(-(x - 1) ** 2 / (sig ** 2 * (1 + 4 * a * t / sig ** 2)))
    err = np.abs(Pn[4, 0, 0, gc.i1:gc.i2 + 1] - 1.0 - g).mean()
    assert err < 2e-4, err


def test_linear_fast_wave_second_order():
    errs = []
    for N in (32, 64, 128):
        gc = P.make_grid(N, 1, 1, dims=1, bc=0)
        amp = 1e-6
        prim, bfld, c = P.linear_wave(gc, "fast", amp=amp)
        s = oracle_sim(dict(Nx=N, Ny=1, Nz=1, dims=1, gam=5. / 3, cour=0.4))
        s.set_state(prim, bfld)
        s.init()
        tend = 1.0 / c  # one crossing of the unit box
        s.advance(tend)
        Pn, _, _ = s.get_state()
        x = gc.lv[0][gc.i1:gc.i2 + 1]
        drho = Pn[0, 0, 0, gc.i1:gc.i2 + 1] - 1.0
        errs.append(np.abs(drho - amp * np.sin(2 * math.pi * (x - c * tend))).mean() / amp)
    order = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(order) > 1.7, (errs, order)


def test_sts_coefficients_rkl2():
    """diffusion.pyx:227-260: RKL2 stage weights; stage count diffusion.pyx:217-224."""
    from oracle import oracle as O
    assert O.get_nsts(1.0, 2.0) == 1
    assert O.get_nsts(1.0, 1.0 / 4.7) == int(0.5 * (math.sqrt(9 + 16 * 4.7) - 1)) + 1
    s = 7
    c = O.get_sts_coeff(s)
    w1 = 4. / (s * s + s - 2)
    assert c[1, 2] == w1 / 3
    for j in range(2, s + 1):
        bj = (j * j + j - 2) / (2 * j * (j + 1))
        bj1 = (1 / 3) if j - 1 < 2 else ((j - 1) ** 2 + (j - 1) - 2) / (2 * (j - 1) * j)
        assert abs(c[j, 0] - (2 * j - 1) / j * bj / bj1) < 1e-15
    # consistency of RKL2: sum of mu + nu + (1 - mu - nu) = 1 trivially; mut > 0
    assert (c[1:, 2] > 0).all()
