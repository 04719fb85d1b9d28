"""The hand-written discrete adjoint (bnz_step_adjoint / bnz_rollout_* and
bonzo_b200.adjoint.rollout) against torch autograd through the FP64 torch
transcription of the step (tests/torch_vl2.py), and against central finite
differences of the device forward on the 256^2, 100-step vortex rollout."""
import math

import numpy as np
import pytest

from helpers import device_ctx, setup_case

pytestmark = pytest.mark.gpu


def _state(case, n, noise=0.0, **kw):
    """Initial state after init (cell B from the faces), as full arrays; with
    noise > 0 every active value is multiplied by (1 + noise * N(0,1)), which
    removes the exact ties (equal wave speeds, equal slopes) of symmetric ICs."""
    import torch
    gc, prim, bfld, opts = setup_case(case, n=n)
    m = dict(rsolver="hlld", limiter="vl", outflow_face_aware=1)
    m.update(kw)
    ref = device_ctx(opts, path="plain", **m)
    ref.set_state(prim, bfld)
    ref.init()
    P0, _, B0 = ref.get_state()
    if noise > 0:
        rng = np.random.default_rng(17)
        P0 = P0 * (1 + noise * rng.normal(size=P0.shape)) + noise * 0.1 * rng.normal(size=P0.shape)
        P0[0] = np.abs(P0[0])
        P0[4] = np.abs(P0[4])
        B0 = B0 * (1 + noise * rng.normal(size=B0.shape))
    ref.set_state(P0, B0)
    dt = ref.new_dt()
    return gc, opts, m, torch.from_numpy(P0[:, 0].copy()), torch.from_numpy(B0[:, 0].copy()), dt


def _rel(a, b):
    s = max(float(b.abs().max()), 1e-300)
    return float((a - b).abs().max()) / s


# The blast's ambient medium is exactly uniform: its faces sit on the HLLD
# region boundary sM = 0, where the derivative depends on the sign rounding
# gives sM; it is checked with noise only.  Likewise the noise-free vortex has
# faces with exactly equal fast speeds on both sides (cfL = cfR): the exact
# build keeps those ties, the fast build's contracted arithmetic can break them
# either way, which moves the derivative of max(cfL, cfR) to the other side.
# Noise-free HLLT therefore runs on the exact build (exact_fp).
@pytest.mark.parametrize("case,n,noise,kw", [
    ("vortex", 24, 0.0, dict(limiter="mc")),
    ("vortex", 24, 1e-3, dict(limiter="vl")),
    ("blast", 24, 1e-3, dict()),
    ("blast", 24, 1e-3, dict(limiter="mc")),
    ("blast_reflect", 20, 1e-3, dict(rsolver="hll")),
    ("mixed_bc", 20, 1e-3, dict(limiter="mm")),
    # constant gravity (both stages' source terms), reflecting walls included
    ("vortex", 24, 0.0, dict(limiter="mc", grav=(0.3, -0.8, 0.1))),
    ("blast", 24, 1e-3, dict(grav=(0.5, -0.5, 0.2))),
    ("blast_reflect", 20, 1e-3, dict(rsolver="hll", grav=(0.0, -1.0, 0.0))),
    # the three-wave HLLT solver
    ("vortex", 24, 0.0, dict(limiter="mc", rsolver="hllt", exact_fp=1)),
    ("vortex", 24, 1e-3, dict(limiter="mc", rsolver="hllt")),
    ("blast", 24, 1e-3, dict(rsolver="hllt")),
    ("mixed_bc", 20, 1e-3, dict(limiter="mm", rsolver="hllt", grav=(0.2, -0.4, 0.0))),
    # slopes projected on the characteristic basis (charact_proj)
    ("vortex", 24, 0.0, dict(limiter="mc", charact_proj=1, exact_fp=1)),
    ("vortex", 24, 1e-3, dict(limiter="mc", charact_proj=1)),
    ("blast", 24, 1e-3, dict(charact_proj=1)),
    ("blast_reflect", 20, 1e-3, dict(rsolver="hll", limiter="mm", charact_proj=1)),
])
def test_step_adjoint_matches_torch_autograd(case, n, noise, kw):
    import torch
    import torch_vl2 as T
    gc, opts, m, P0, B0, dt = _state(case, n, noise=noise, **kw)
    G = T.Grid(gc, face_aware=True, device="cuda")
    p = P0.cuda().requires_grad_(True)
    b = B0.cuda().requires_grad_(True)
    tp, tb = T.step(G, p, b, dt, rs=m["rsolver"], lim=m["limiter"], grav=m.get("grav"),
                    charact=bool(m.get("charact_proj")))
    gen = torch.Generator(device="cpu").manual_seed(5)
    gp = torch.randn(tp.shape, generator=gen, dtype=torch.float64).cuda()
    gb = torch.randn(tb.shape, generator=gen, dtype=torch.float64).cuda()
    ap, ab = torch.autograd.grad((tp * gp).sum() + (tb * gb).sum(), (p, b))

    eng = device_ctx(opts, path="fused", **m)
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
    shp = (1,) + tuple(P0.shape[1:])
    P = P0.reshape((9,) + shp).cuda().contiguous()
    B = B0.reshape((3,) + shp).cuda().contiguous()
    gp4 = gp.reshape(P.shape).contiguous()
    gb4 = gb.reshape(B.shape).contiguous()
    op, ob = torch.empty_like(P), torch.empty_like(B)
    eng.step_adjoint(dt, P.data_ptr(), B.data_ptr(), gp4.data_ptr(), gb4.data_ptr(), op.data_ptr(), ob.data_ptr())
    torch.cuda.synchronize()
    # the step's forward agrees with the transcription
    fp, fb = torch.empty_like(P), torch.empty_like(B)
    eng.get_state_device(fp.data_ptr(), fb.data_ptr())
    torch.cuda.synchronize()
    assert _rel(fp[:, 0], tp.detach()) < 1e-12
    assert _rel(fb[:, 0], tb.detach()) < 1e-12
    # gradients: tolerance 1e-9 of the largest entry, per field
    for v in range(9):
        assert _rel(op[v, 0], ap[v]) < 1e-9, (v, _rel(op[v, 0], ap[v]))
    for v in range(3):
        assert _rel(ob[v, 0], ab[v]) < 1e-9, (v, _rel(ob[v, 0], ab[v]))


@pytest.mark.parametrize("nsteps,every,extra", [
    (7, 3, {}), (6, 6, {}), (5, 1, {}),
    (6, 4, dict(grav=(0.2, -0.6, 0.0))),
    # HLLT on the exact build (the vortex's exact wave-speed ties, see above)
    (5, 2, dict(grav=(0.0, -0.5, 0.0), rsolver="hllt", exact_fp=1)),
    (4, 2, dict(charact_proj=1, exact_fp=1)),
])
def test_rollout_adjoint_matches_torch_autograd(nsteps, every, extra):
    import torch
    import torch_vl2 as T
    from bonzo_b200.adjoint import rollout
    kw = dict(limiter="mc")
    kw.update(extra)
    rs, grav = kw.get("rsolver", "hlld"), kw.get("grav")
    gc, opts, m, P0, B0, dt = _state("vortex_pert", 32, **kw)
    dt = 0.5 * dt
    G = T.Grid(gc, face_aware=True, device="cuda")
    gen = torch.Generator(device="cpu").manual_seed(9)
    target = (P0[0] + 0.1 * torch.randn(P0[0].shape, generator=gen, dtype=torch.float64)).cuda()
    # torch autograd through the transcription
    p = P0.cuda().requires_grad_(True)
    b = B0.cuda().requires_grad_(True)
    x, y = p, b
    for _ in range(nsteps):
        x, y = T.step(G, x, y, dt, rs=rs, lim="mc", grav=grav, charact=bool(kw.get("charact_proj")))
    loss_t = ((x[0] - target) ** 2).sum()
    ap, ab = torch.autograd.grad(loss_t, (p, b))
    # the adjoint through the autograd wrapper
    eng = device_ctx(opts, path="fused", **m)
    shp = (9, 1) + tuple(P0.shape[1:])
    p4 = P0.reshape(shp).cuda().requires_grad_(True)
    b4 = B0.reshape((3,) + shp[1:]).cuda().requires_grad_(True)
    xp, xb = rollout(p4, b4, eng, nsteps, dt, checkpoint_every=every)
    loss = ((xp[0, 0] - target) ** 2).sum()
    loss.backward()
    assert abs(loss.item() - loss_t.item()) <= 1e-12 * abs(loss_t.item())
    for v in range(9):
        assert _rel(p4.grad[v, 0], ap[v]) < 1e-9, (v, _rel(p4.grad[v, 0], ap[v]))
    for v in range(3):
        assert _rel(b4.grad[v, 0], ab[v]) < 1e-9, (v, _rel(b4.grad[v, 0], ab[v]))


def _vortex_ic(gc, v, az, gam=5.0 / 3.0, beta=4 * math.pi):
    """Differentiable vortex initial state from active-cell velocities v (2, Ny, Nx)
    and the corner potential az (Ny+1, Nx+1): faces as corner differences, cell
    B as face averages (the state init would produce), ghosts zero."""
    import torch
    i1, i2, j1, j2 = gc.i1, gc.i2, gc.j1, gc.j2
    dx, dy = gc.dlf[0][i1], gc.dlf[1][j1]
    sb = math.sqrt(beta)
    prim = torch.zeros((9, 1) + tuple(gc.shape[1:]), dtype=torch.float64, device="cuda")
    bfld = torch.zeros((3, 1) + tuple(gc.shape[1:]), dtype=torch.float64, device="cuda")
    bx = (az[1:, :] - az[:-1, :]) / dy / sb
    by = -(az[:, 1:] - az[:, :-1]) / dx / sb
    prim[0, 0, j1:j2 + 1, i1:i2 + 1] = gam * gam
    prim[4, 0, j1:j2 + 1, i1:i2 + 1] = gam
    prim[1, 0, j1:j2 + 1, i1:i2 + 1] = v[0]
    prim[2, 0, j1:j2 + 1, i1:i2 + 1] = v[1]
    prim[6, 0, j1:j2 + 1, i1:i2 + 1] = 0.5 * (bx[:, :-1] + bx[:, 1:])
    prim[7, 0, j1:j2 + 1, i1:i2 + 1] = 0.5 * (by[:-1, :] + by[1:, :])
    bfld[0, 0, j1:j2 + 1, i1:i2 + 2] = bx
    bfld[1, 0, j1:j2 + 2, i1:i2 + 1] = by
    return prim, bfld


def test_rollout_gradient_matches_central_differences_256():
    """The adjoint-rollout check: 256^2 periodic vortex with a seeded smooth
    perturbation, 100 steps of dt = 1e-4 (VL2 + PLM(mc) + HLLD + CT), loss =
    squared misfit of the final density to a seeded smooth target; gradient with
    respect to the initial velocity and Az (device adjoint, checkpoint every 10
    steps) against central differences (eps = 1e-6) along 8 seeded directions.

    The discrete step is piecewise smooth: limiter cases and Riemann fan regions
    switch within 1e-6 of the state at many cells (the vortex starts with
    uniform density and pressure), so plain differences do not converge.  The
    differences are therefore taken with every branch decision frozen at the
    base point (recorded and replayed by the torch transcription of the step,
    run on the GPU), which makes the map smooth; its derivative at the base
    point is the one the adjoint computes."""
    import torch
    import torch_vl2 as T
    from bonzo_b200 import problems as P
    from bonzo_b200.adjoint import rollout
    n, nsteps, dt = 256, 100, 1e-4
    gc = P.make_grid(n, n, 1, dims=2, bc=0)
    prim0, bfld0 = P.otvortex(gc, pert_amp=1e-2, seed=3)
    i1, i2, j1, j2 = gc.i1, gc.i2, gc.j1, gc.j2
    v0 = torch.from_numpy(prim0[1:3, 0, j1:j2 + 1, i1:i2 + 1].copy()).cuda()
    dx, dy = gc.dlf[0][i1], gc.dlf[1][j1]
    # recover Az on the corners from the faces (Az(j1, i) fixed by the x-face
    # sums along y; the potential is defined up to a constant)
    sb = math.sqrt(4 * math.pi)
    bx = bfld0[0, 0, j1:j2 + 1, i1:i2 + 2]
    by = bfld0[1, 0, j1:j2 + 2, i1:i2 + 1]
    az = np.zeros((n + 1, n + 1))
    az[0, 1:] = -np.cumsum(by[0, :]) * dx * sb
    az[1:, :] = az[0:1, :] + np.cumsum(bx, axis=0) * dy * sb
    az0 = torch.from_numpy(az).cuda()
    x = gc.lv[0][i1:i2 + 1]
    y = gc.lv[1][j1:j2 + 1]
    X, Y = np.meshgrid(x, y)
    target = torch.from_numpy((5. / 3) ** 2 * (1 + 0.05 * np.sin(2 * math.pi * X) * np.cos(4 * math.pi * Y))).cuda()
    opts = dict(Nx=n, Ny=n, Nz=1, dims=2, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4,
                rsolver="hlld", limiter="mc", path="fused")
    eng = device_ctx(opts)

    # gradient through the device adjoint
    v = v0.clone().requires_grad_(True)
    a = az0.clone().requires_grad_(True)
    p, b = _vortex_ic(gc, v, a)
    xp, _ = rollout(p, b, eng, nsteps, dt, checkpoint_every=10)
    L = ((xp[0, 0, j1:j2 + 1, i1:i2 + 1] - target) ** 2).sum()
    L.backward()
    gv, ga = v.grad.clone(), a.grad.clone()

    # branch-frozen central differences of the transcription
    G = T.Grid(gc, face_aware=True, device="cuda")

    def loss_t(vv, aa):
        pp, bb = _vortex_ic(gc, vv, aa)
        xx, yy = pp[:, 0], bb[:, 0]
        for _ in range(nsteps):
            xx, yy = T.step(G, xx, yy, dt, rs="hlld", lim="mc")
        return float(((xx[0, j1:j2 + 1, i1:i2 + 1] - target) ** 2).sum())

    try:
        with torch.no_grad():
            T.BRANCHES.record()
            L0 = loss_t(v0, az0)
            assert abs(L0 - float(L.detach())) <= 1e-12 * abs(L0)
            gen = torch.Generator(device="cpu").manual_seed(2026)
            eps = 1e-6
            worst = 0.0
            for _ in range(8):
                dv = torch.randn(v0.shape, generator=gen, dtype=torch.float64).cuda()
                da = 0.1 * torch.randn(az0.shape, generator=gen, dtype=torch.float64).cuda()
                T.BRANCHES.replay()
                lp = loss_t(v0 + eps * dv, az0 + eps * da)
                T.BRANCHES.replay()
                lm = loss_t(v0 - eps * dv, az0 - eps * da)
                fd = (lp - lm) / (2 * eps)
                ad = float((gv * dv).sum() + (ga * da).sum())
                worst = max(worst, abs(fd - ad) / abs(ad))
    finally:
        T.BRANCHES.off()
    assert worst <= 1e-6, worst


def _c3_setup(n, seed=3):
    """The adjoint configuration's state at n^2: the periodic vortex plus a
    seeded smooth perturbation (Fourier modes |k| <= 4, amplitude 1e-2) on v
    and Az, a seeded smooth density target, the corner potential recovered
    from the faces."""
    import torch
    from bonzo_b200 import problems as P
    gc = P.make_grid(n, n, 1, dims=2, bc=0)
    prim0, bfld0 = P.otvortex(gc, pert_amp=1e-2, seed=seed)
    i1, i2, j1, j2 = gc.i1, gc.i2, gc.j1, gc.j2
    v0 = torch.from_numpy(prim0[1:3, 0, j1:j2 + 1, i1:i2 + 1].copy()).cuda()
    dx, dy = gc.dlf[0][i1], gc.dlf[1][j1]
    sb = math.sqrt(4 * math.pi)
    bx = bfld0[0, 0, j1:j2 + 1, i1:i2 + 2]
    by = bfld0[1, 0, j1:j2 + 2, i1:i2 + 1]
    az = np.zeros((n + 1, n + 1))
    az[0, 1:] = -np.cumsum(by[0, :]) * dx * sb
    az[1:, :] = az[0:1, :] + np.cumsum(bx, axis=0) * dy * sb
    x = gc.lv[0][i1:i2 + 1]
    y = gc.lv[1][j1:j2 + 1]
    X, Y = np.meshgrid(x, y)
    target = torch.from_numpy((5. / 3) ** 2 * (1 + 0.05 * np.sin(2 * math.pi * X) * np.cos(4 * math.pi * Y))).cuda()
    return gc, v0, torch.from_numpy(az).cuda(), target


def test_rollout_adjoint_64_matches_torch_autograd():
    """The adjoint configuration at 64 x 64 as it is worded: 100 steps of
    dt = 1e-4 (VL2 + PLM(mc) + HLLD + CT), checkpoint every 10 steps, loss =
    squared misfit of the final density; the gradient with respect to the
    initial velocity and Az from the device adjoint against torch autograd
    through the FP64 torch transcription of the step."""
    import torch
    import torch_vl2 as T
    from bonzo_b200.adjoint import rollout
    n, nsteps, dt = 64, 100, 1e-4
    gc, v0, az0, target = _c3_setup(n)
    i1, i2, j1, j2 = gc.i1, gc.i2, gc.j1, gc.j2
    opts = dict(Nx=n, Ny=n, Nz=1, dims=2, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4,
                rsolver="hlld", limiter="mc", path="fused")
    eng = device_ctx(opts)
    v = v0.clone().requires_grad_(True)
    a = az0.clone().requires_grad_(True)
    p, b = _vortex_ic(gc, v, a)
    xp, _ = rollout(p, b, eng, nsteps, dt, checkpoint_every=10)
    L = ((xp[0, 0, j1:j2 + 1, i1:i2 + 1] - target) ** 2).sum()
    L.backward()
    G = T.Grid(gc, face_aware=True, device="cuda")
    vt = v0.clone().requires_grad_(True)
    at = az0.clone().requires_grad_(True)
    pt, bt = _vortex_ic(gc, vt, at)
    xx, yy = pt[:, 0], bt[:, 0]
    for _ in range(nsteps):
        xx, yy = T.step(G, xx, yy, dt, rs="hlld", lim="mc")
    Lt = ((xx[0, j1:j2 + 1, i1:i2 + 1] - target) ** 2).sum()
    Lt.backward()
    assert abs(float(L.detach()) - float(Lt.detach())) <= 1e-12 * abs(float(Lt.detach()))
    assert _rel(v.grad, vt.grad) < 1e-9, _rel(v.grad, vt.grad)
    assert _rel(a.grad, at.grad) < 1e-9, _rel(a.grad, at.grad)


@pytest.mark.parametrize("nsteps", [1, 3])
def test_adjoint_dot_product(nsteps):
    """<J v, w> = <v, J^T w> for the map of nsteps steps at a perturbed vortex
    state: J v by forward-mode differentiation of the torch transcription
    (torch.func.jvp), J^T w by the device's hand-written reverse pass -- two
    independent derivative implementations."""
    import torch
    import torch_vl2 as T
    gc, opts, m, P0, B0, dt = _state("vortex_pert", 48, limiter="mc")
    G = T.Grid(gc, face_aware=True, device="cuda")
    gen = torch.Generator(device="cpu").manual_seed(11)
    a = (slice(None),) + tuple(gc.active[1:])
    vp = torch.zeros(P0.shape, dtype=torch.float64)
    vb = torch.zeros(B0.shape, dtype=torch.float64)
    vp[a] = torch.randn(vp[a].shape, generator=gen, dtype=torch.float64)
    vb[a] = torch.randn(vb[a].shape, generator=gen, dtype=torch.float64)
    vp, vb = vp.cuda(), vb.cuda()

    def f(p, b):
        for _ in range(nsteps):
            p, b = T.step(G, p, b, dt, rs="hlld", lim="mc")
        return p, b

    out, (jp, jb) = torch.func.jvp(f, (P0.cuda(), B0.cuda()), (vp, vb))
    wp = torch.randn(out[0].shape, generator=gen, dtype=torch.float64).cuda()
    wb = torch.randn(out[1].shape, generator=gen, dtype=torch.float64).cuda()
    lhs = float((jp * wp).sum() + (jb * wb).sum())
    # J^T w on the device: the rollout adjoint (tape of every step)
    eng = device_ctx(opts, path="fused", **m)
    eng.set_stream(torch.cuda.current_stream().cuda_stream)
    shp = (1,) + tuple(P0.shape[1:])
    P = P0.reshape((9,) + shp).cuda().contiguous()
    B = B0.reshape((3,) + shp).cuda().contiguous()
    eng.set_state_device(P.data_ptr(), B.data_ptr())
    eng.rollout_forward(nsteps, dt, 1)
    gp4, gb4 = wp.reshape(P.shape).contiguous(), wb.reshape(B.shape).contiguous()
    op, ob = torch.empty_like(P), torch.empty_like(B)
    eng.rollout_adjoint(gp4.data_ptr(), gb4.data_ptr(), op.data_ptr(), ob.data_ptr())
    torch.cuda.synchronize()
    rhs = float((vp * op[:, 0]).sum() + (vb * ob[:, 0]).sum())
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def test_adjoint_rejects_turbulence_driving():
    """The driving force is a random field advanced every step that the tape
    does not keep: the adjoint refuses it on the host, before any launch."""
    from bonzo_b200 import _lib
    gc, prim, bfld, opts = setup_case("vortex", n=16)
    eng = device_ctx(opts, path="fused", rsolver="hlld", limiter="mc", drive_f0=0.5, drive_tau=1.0, drive_nmod=1)
    eng.set_state(prim, bfld)
    eng.init()
    with pytest.raises(_lib.BnzError) as e:
        eng.rollout_forward(3, 1e-4, 1)
    assert e.value.code == _lib.BNZ_ERR_UNSUPPORTED and "driving" in str(e.value)
