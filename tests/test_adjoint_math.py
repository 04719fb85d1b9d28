"""Pointwise VJPs of the adjoint (bonzo_b200/csrc/bnz_adjoint_math.h) against
central finite differences of the forward per-point math (bnz_device.cuh), both
compiled for the host from the shipped headers (tests/adjoint_cpu/adjmath.cpp).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "adjoint_cpu", "adjmath.cpp")
OUT = os.path.join(HERE, "adjoint_cpu", "_build", "libadjmath.so")
GAM = 5.0 / 3.0


@pytest.fixture(scope="module")
def lib():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", OUT, SRC],
                   check=True)
    L = C.CDLL(OUT)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.t_flux.argtypes = [C.c_int, dp, dp, C.c_double, dp]
    L.t_vjp_flux.argtypes = [C.c_int, dp, dp, C.c_double, dp, dp, dp]
    L.t_hlld_region.argtypes = [dp, dp, C.c_double]
    L.t_hllt_region.argtypes = [dp, dp, C.c_double]
    L.t_cons2prim.argtypes = [dp, C.c_double, dp]
    L.t_prim2cons.argtypes = [dp, C.c_double, dp]
    L.t_vjp_cons2prim.argtypes = [dp, dp, C.c_double, dp]
    L.t_vjp_prim2cons.argtypes = [dp, dp, C.c_double, dp]
    L.t_plm.argtypes = [C.c_int, dp, dp]
    L.t_vjp_plm.argtypes = [C.c_int, dp, C.c_double, C.c_double, dp]
    L.t_slopes_char.argtypes = [C.c_int, C.c_int, dp, dp, dp, C.c_double, dp]
    L.t_vjp_slopes_char.argtypes = [C.c_int, dp, dp, dp, C.c_double, dp, dp, dp, dp]
    return L


def states(rng, n):
    """Seeded face states; every fourth pair streams supersonically (fan regions
    1 / 6), every fifth has a strong normal field (regions 2 / 5 open up),
    every ninth has a zero normal field."""
    out = []
    for q in range(n):
        w = np.zeros((2, 9))
        w[:, 0] = rng.uniform(0.2, 3.0, 2)
        w[:, 1:4] = rng.normal(0, 1.0, (2, 3))
        w[:, 4] = rng.uniform(0.1, 3.0, 2)
        w[:, 5] = rng.uniform(0, 1, 2)
        w[:, 7:9] = rng.normal(0, 1, (2, 2))
        w[:, 6] = rng.normal(0, 1)
        if q % 4 == 1:
            w[:, 1] = (6.0 if q % 8 == 1 else -6.0) + rng.normal(0, 0.5, 2)
        if q % 5 == 2:
            w[:, 6] = 3.0 * np.sign(w[0, 6])
            w[:, 1] += 1.5 if q % 10 == 2 else -1.5
        if q % 9 == 4:
            w[:, 6] = 0.0
        out.append(w)
    return out


def fd_flux(L, rs, wL, wR, fb, h):
    """Central differences of fb . flux: 17 entries, wL (the shared normal field
    at BX) then the 8 tangential entries of wR."""
    def phi(l, r):
        f = np.zeros(9)
        L.t_flux(rs, l, r, GAM, f)
        return float(fb @ f)
    g = []
    for side in (0, 1):
        for k in range(9):
            if side == 1 and k == 6:
                continue
            base = wL if side == 0 else wR
            s = h * max(1.0, abs(base[k]))
            la, lb, ra, rb = wL.copy(), wL.copy(), wR.copy(), wR.copy()
            if side == 0 or k == 6:
                la[k] += s
                lb[k] -= s
            if side == 1 or k == 6:
                ra[k] += s
                rb[k] -= s
            g.append((phi(la, ra) - phi(lb, rb)) / (2 * s))
    return np.array(g)


@pytest.mark.parametrize("rs", [0, 2, 3], ids=["hll", "hlld", "hllt"])
def test_riemann_vjp_matches_finite_differences(lib, rs):
    rng = np.random.default_rng(7 + rs)
    ok = skipped = 0
    regions = set()
    for w in states(rng, 160):
        wL, wR = w[0].copy(), w[1].copy()
        wR[6] = wL[6]
        fb = rng.normal(0, 1, 9)
        fb[6] = 0.0
        vL, vR = np.zeros(9), np.zeros(9)
        lib.t_vjp_flux(rs, wL, wR, GAM, fb, vL, vR)
        v = np.concatenate([vL[:6], [vL[6] + vR[6]], vL[7:], vR[:6], vR[7:]])
        g1 = fd_flux(lib, rs, wL, wR, fb, 1e-6)
        g2 = fd_flux(lib, rs, wL, wR, fb, 1e-7)
        scale = max(1.0, np.max(np.abs(g1)))
        if np.max(np.abs(g1 - g2)) > 1e-5 * scale:
            skipped += 1  # a kink (fan region / wave-speed switch) within the FD stencil
            continue
        assert np.max(np.abs(v - g1)) <= 2e-6 * scale, (v - g1, wL, wR)
        ok += 1
        if rs == 2:
            regions.add(lib.t_hlld_region(wL, wR, GAM))
        if rs == 3:
            regions.add(lib.t_hllt_region(wL, wR, GAM))
    assert skipped <= 8, skipped
    assert ok >= 140
    if rs == 2:
        assert regions == {1, 2, 3, 4, 5, 6}, regions
    if rs == 3:
        assert regions == {1, 2, 3, 4, 5}, regions


def test_eos_vjps_match_finite_differences(lib):
    rng = np.random.default_rng(3)
    for w in states(rng, 40):
        w0 = w[0]
        u0 = np.zeros(9)
        lib.t_prim2cons(w0, GAM, u0)
        # cons2prim: d(wb . w(u)) / du
        wb = rng.normal(0, 1, 9)
        ub = np.zeros(9)
        lib.t_vjp_cons2prim(w0, wb, GAM, ub)
        g = np.zeros(9)
        for k in range(9):
            s = 1e-6 * max(1.0, abs(u0[k]))
            a, b = u0.copy(), u0.copy()
            a[k] += s
            b[k] -= s
            wa, wbb = np.zeros(9), np.zeros(9)
            lib.t_cons2prim(a, GAM, wa)
            lib.t_cons2prim(b, GAM, wbb)
            g[k] = wb @ (wa - wbb) / (2 * s)
        assert np.allclose(ub, g, rtol=1e-6, atol=1e-7)
        # prim2cons
        ubar = rng.normal(0, 1, 9)
        wbar = np.zeros(9)
        lib.t_vjp_prim2cons(w0, ubar, GAM, wbar)
        for k in range(9):
            s = 1e-6 * max(1.0, abs(w0[k]))
            a, b = w0.copy(), w0.copy()
            a[k] += s
            b[k] -= s
            ua, ubb = np.zeros(9), np.zeros(9)
            lib.t_prim2cons(a, GAM, ua)
            lib.t_prim2cons(b, GAM, ubb)
            g[k] = ubar @ (ua - ubb) / (2 * s)
        assert np.allclose(wbar, g, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("lim", [0, 1, 2], ids=["vl", "mc", "mm"])
def test_plm_vjp_matches_finite_differences(lib, lim):
    rng = np.random.default_rng(11 + lim)
    n = 0
    for _ in range(300):
        c4 = np.cumsum(rng.normal(0, 1, 4))
        bL, bR = rng.normal(0, 1, 2)
        cb = np.zeros(4)
        lib.t_vjp_plm(lim, c4, bL, bR, cb)
        g = np.zeros(4)
        for k in range(4):
            s = 1e-7
            a, b = c4.copy(), c4.copy()
            a[k] += s
            b[k] -= s
            oa, ob = np.zeros(2), np.zeros(2)
            lib.t_plm(lim, a, oa)
            lib.t_plm(lim, b, ob)
            g[k] = (bL * (oa[0] - ob[0]) + bR * (oa[1] - ob[1])) / (2 * s)
        # skip stencils within the FD step of a limiter switch
        d = np.diff(c4)
        if np.min(np.abs(d)) < 1e-5 or abs(2 * d[0] - 0.5 * (d[0] + d[1])) < 1e-5 or \
                abs(2 * d[1] - 0.5 * (d[1] + d[2])) < 1e-5 or abs(d[0] - d[1]) < 1e-5 or \
                abs(d[1] - d[2]) < 1e-5 or abs(2 * d[1] - 0.5 * (d[0] + d[1])) < 1e-5 or \
                abs(2 * d[0] - 0.5 * (d[0] + d[1])) < 1e-5 or abs(2 * d[2] - 0.5 * (d[1] + d[2])) < 1e-5:
            continue
        assert np.allclose(cb, g, rtol=1e-6, atol=1e-7), (lim, c4, cb, g)
        n += 1
    assert n > 250


@pytest.mark.parametrize("lim", [0, 1, 2], ids=["vl", "mc", "mm"])
def test_characteristic_slope_vjp_matches_finite_differences(lib, lim):
    """The projected slope (prim2char, limiter, char2prim) of three cells: the
    adjoint header's forward equals the device forward, and its VJP matches
    central differences over all 27 inputs, the eigen-system coefficients'
    dependence on the centre cell included."""
    rng = np.random.default_rng(23 + lim)
    ok = skipped = 0
    for w in states(rng, 60):
        wc = w[0].copy()
        if wc[6] == 0.0:
            continue  # sgn(bx) switches at bx = 0: a kink both FD steps straddle alike
        wm = wc + 0.2 * rng.normal(size=9)
        wp = wc + 0.2 * rng.normal(size=9)
        for a in (wm, wp):
            a[0] = abs(a[0]) + 0.1
            a[4] = abs(a[4]) + 0.1
        d0, d1 = np.zeros(9), np.zeros(9)
        lib.t_slopes_char(0, lim, wm, wc, wp, GAM, d0)
        lib.t_slopes_char(1, lim, wm, wc, wp, GAM, d1)
        assert np.allclose(d0, d1, rtol=1e-12, atol=1e-13), (d0, d1)
        db = rng.normal(size=9)
        bm, bc, bp = np.zeros(9), np.zeros(9), np.zeros(9)
        lib.t_vjp_slopes_char(lim, wm, wc, wp, GAM, db, bm, bc, bp)
        v = np.concatenate([bm, bc, bp])

        def fd(h):
            g = np.zeros(27)
            for t in range(27):
                arrs = [wm.copy(), wc.copy(), wp.copy()]
                base = arrs[t // 9][t % 9]
                s_ = h * max(1.0, abs(base))
                out = []
                for sign in (1, -1):
                    a = [x.copy() for x in arrs]
                    a[t // 9][t % 9] = base + sign * s_
                    d = np.zeros(9)
                    lib.t_slopes_char(0, lim, a[0], a[1], a[2], GAM, d)
                    out.append(db @ d)
                g[t] = (out[0] - out[1]) / (2 * s_)
            return g
        g1, g2 = fd(1e-6), fd(1e-7)
        scale = max(1.0, np.max(np.abs(g1)))
        if np.max(np.abs(g1 - g2)) > 1e-5 * scale:
            skipped += 1  # a limiter or eigen-system case switch within the stencil
            continue
        assert np.max(np.abs(v - g1)) <= 2e-6 * scale, (lim, v - g1)
        ok += 1
    assert ok >= 45, (ok, skipped)
