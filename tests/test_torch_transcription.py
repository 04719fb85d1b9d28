"""The torch transcription of the step (tests/torch_vl2.py), the checker of
the adjoint, pinned against the oracle's step and self-checked: with branch
decisions frozen, its central differences converge to its autograd gradient."""

import numpy as np
import pytest

from helpers import oracle_sim, setup_case


@pytest.mark.parametrize("case,n,kw", [
    ("vortex", 20, dict(limiter="mc")),
    ("blast", 20, dict()),
    ("blast_reflect", 16, dict(rsolver="hll")),
    ("mixed_bc", 16, dict(limiter="mm")),
    ("blast", 16, dict(grav=(0.3, -1.2, 0.05))),
    ("vortex", 16, dict(limiter="mc", rsolver="hll", grav=(-0.7, 0.4, 0.0))),
    ("vortex", 20, dict(limiter="mc", rsolver="hllt")),
    ("blast", 20, dict(rsolver="hllt")),
    ("mixed_bc", 16, dict(limiter="mm", rsolver="hllt")),
    ("vortex_pert", 20, dict(limiter="mc", charact_proj=1)),
    ("blast", 20, dict(charact_proj=1)),
    ("blast_reflect", 16, dict(limiter="mm", rsolver="hll", charact_proj=1)),
])
def test_transcription_matches_oracle_step(case, n, kw):
    import torch
    import torch_vl2 as T
    gc, prim, bfld, opts = setup_case(case, n=n)
    m = dict(rsolver="hlld", limiter="vl", outflow_face_aware=1)
    m.update(kw)
    o = oracle_sim(opts, **m)
    o.set_state(prim, bfld)
    o.init()
    P0, _, B0 = o.get_state()
    dt = o.new_dt()
    o.step(dt)
    P1, _, B1 = o.get_state()
    G = T.Grid(gc, face_aware=True)
    tp, tb = T.step(G, torch.from_numpy(P0[:, 0].copy()), torch.from_numpy(B0[:, 0].copy()), dt,
                    rs=m["rsolver"], lim=m["limiter"], grav=m.get("grav"), charact=bool(m.get("charact_proj")))
    for a, b in ((tp.numpy(), P1[:, 0]), (tb.numpy(), B1[:, 0])):
        for v in range(a.shape[0]):
            s = max(np.abs(b[v]).max(), 1e-300)
            assert np.abs(a[v] - b[v]).max() <= 1e-13 * s


@pytest.mark.parametrize("charact", [False, True], ids=["plm", "charact_proj"])
def test_branch_frozen_differences_converge_to_autograd(charact):
    import torch
    import torch_vl2 as T
    from bonzo_b200 import problems as P
    n, nsteps, dt = 16, 4, 2e-4
    gc = P.make_grid(n, n, 1, dims=2, bc=0)
    prim0, bfld0 = P.otvortex(gc, pert_amp=1e-2, seed=1)
    i1, i2, j1, j2 = gc.i1, gc.i2, gc.j1, gc.j2
    prim0[6, 0, j1:j2 + 1, i1:i2 + 1] = 0.5 * (bfld0[0, 0, j1:j2 + 1, i1:i2 + 1] + bfld0[0, 0, j1:j2 + 1, i1 + 1:i2 + 2])
    prim0[7, 0, j1:j2 + 1, i1:i2 + 1] = 0.5 * (bfld0[1, 0, j1:j2 + 1, i1:i2 + 1] + bfld0[1, 0, j1 + 1:j2 + 2, i1:i2 + 1])
    G = T.Grid(gc)
    p0 = torch.from_numpy(prim0[:, 0].copy())
    b0 = torch.from_numpy(bfld0[:, 0].copy())
    rng = np.random.default_rng(0)
    tgt = torch.from_numpy(rng.normal(size=p0[0].shape))

    def L(p, b):
        x, y = p, b
        for _ in range(nsteps):
            x, y = T.step(G, x, y, dt, rs="hlld", lim="mc", charact=charact)
        return ((x[0] - tgt) ** 2).sum() + (x[1] ** 2).sum()

    p = p0.clone().requires_grad_(True)
    b = b0.clone().requires_grad_(True)
    try:
        T.BRANCHES.record()
        L(p, b).backward()
        for _ in range(3):
            dp = torch.zeros_like(p0)
            dp[1:3] = torch.from_numpy(rng.normal(size=dp[1:3].shape))
            db = torch.from_numpy(0.1 * rng.normal(size=b0.shape))
            ad = float((p.grad * dp).sum() + (b.grad * db).sum())
            eps = 1e-6
            with torch.no_grad():
                T.BRANCHES.replay()
                lp = float(L(p0 + eps * dp, b0 + eps * db))
                T.BRANCHES.replay()
                lm = float(L(p0 - eps * dp, b0 - eps * db))
            assert abs((lp - lm) / (2 * eps) - ad) <= 1e-6 * abs(ad)
    finally:
        T.BRANCHES.off()
