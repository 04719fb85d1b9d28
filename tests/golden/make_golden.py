"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Run where the reference tree is available (it builds oracle/_ref from the
reference's C sources first):

    python tests/golden/make_golden.py

Fixtures:
  kernels_mhd.npz    the reference's hll/hllt/hlld_flux, cons2prim_1,
                     prim2cons_1, fms and reconstr_const/reconstr_linear
                     (with and without characteristic projection) on seeded
                     inputs, including every HLLD wave-fan region and Bx = 0.
  kernels_hydro.npz  the hydro build (MFIELD=0): hll/hllc/hllt_flux and
                     reconstr_linear.
  steps.npz          whole VL2 steps of the oracle driver running the
                     reference's compiled Riemann and reconstruction kernels:
                     initial state, per-step dt and the state after the steps
                     for a 2D periodic vortex, a 2D outflow blast, a 3D
                     periodic turbulence box and a 3D conduction box.
The tests compare the oracle's restated kernels and the device kernels with
these arrays; nothing here is needed at test time except the .npz files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def riemann_inputs(rng, n, nm=9, mhd=True):
    wl = np.zeros((nm, n))
    wr = np.zeros((nm, n))
    for w in (wl, wr):
        w[0] = rng.uniform(0.1, 3.0, n)
        w[1:4] = rng.normal(0, 1.5, (3, n))
        w[4] = rng.uniform(0.05, 3.0, n)
        w[5] = rng.uniform(0, 1, n)
        if mhd:
            w[6:9] = rng.normal(0, 1, (3, n))
    bx = rng.normal(0, 1, n) if mhd else np.zeros(n)
    if mhd:
        bx[::9] = 0.0  # degenerate normal field (sgn(bx) = 0 branch)
        # supersonic left / right streams (fan entirely to one side)
        wl[1, 1::13] = wr[1, 1::13] = 8.0
        wl[1, 2::13] = wr[1, 2::13] = -8.0
    return wl, wr, bx


def main():
    from oracle import build as ob
    from oracle import build_ref as br
    from oracle import oracle as O
    ob.build(quiet=True)
    if not br.build(quiet=True):
        raise SystemExit("reference sources not found; cannot make golden vectors")
    rng = np.random.default_rng(20261203)
    gam = 5.0 / 3.0
    out = {"gam": gam}
    n = 800
    for rs in ("hll", "hllt", "hlld"):
        wl, wr, bx = riemann_inputs(rng, n)
        out[rs + "_wl"], out[rs + "_wr"], out[rs + "_bx"] = wl, wr, bx
        out[rs + "_flux"] = O.ref_flux_flat(rs, wl, wr, bx, gam)
    w = np.zeros((9, n))
    w[0] = rng.uniform(0.1, 3, n)
    w[1:4] = rng.normal(0, 1, (3, n))
    w[4] = rng.uniform(0.05, 3, n)
    w[5] = rng.uniform(0, 1, n)
    w[6:9] = rng.normal(0, 1, (3, n))
    out["eos_w"] = w
    out["eos_u"] = O.ref_row_eos("prim2cons_1", w, gam)
    out["eos_w_back"] = O.ref_row_eos("cons2prim_1", out["eos_u"], gam)
    out["fms"] = np.array([O.ref_fms(w[:, q], gam) for q in range(n)])
    row = np.cumsum(rng.normal(0, 0.2, (9, 160)), axis=1)
    row[0] = np.abs(row[0]) + 0.5
    row[4] = np.abs(row[4]) + 0.5
    out["rc_w"] = row
    for fn, order in (("reconstr_const", 0), ("reconstr_linear", 1)):
        for cp in (0, 1):
            if order == 0 and cp:
                continue
            wl, wr = O.reconstr_with(fn, order, row, gam, use_ref=True, char_proj=cp)
            out["rc_%s_cp%d_wl" % (fn, cp)] = wl
            out["rc_%s_cp%d_wr" % (fn, cp)] = wr
    np.savez_compressed(os.path.join(HERE, "kernels_mhd.npz"), **out)

    outh = {"gam": 1.4}
    for rs in ("hll", "hllc", "hllt"):
        wl, wr, bx = riemann_inputs(rng, n, nm=6, mhd=False)
        outh[rs + "_wl"], outh[rs + "_wr"], outh[rs + "_bx"] = wl, wr, bx
        outh[rs + "_flux"] = O.ref_flux_flat(rs, wl, wr, bx, 1.4, hydro=True)
    rowh = row[:6].copy()
    outh["rc_w"] = rowh
    wl, wr = O.reconstr_with("reconstr_linear", 1, rowh, 1.4, use_ref=True, hydro=True)
    outh["rc_wl"], outh["rc_wr"] = wl, wr
    np.savez_compressed(os.path.join(HERE, "kernels_hydro.npz"), **outh)

    from helpers import setup_case, oracle_sim
    steps = {}
    for case, n_, nsteps in (("vortex", 16, 3), ("blast", 16, 3), ("turb3d", 6, 2), ("cond3d", 6, 2)):
        gc, prim, bfld, opts = setup_case(case, n=n_)
        sim = oracle_sim(opts, use_ref_kernels=True, rsolver="hlld", limiter="vl")
        sim.set_state(prim, bfld)
        sim.init()
        dts = []
        for _ in range(nsteps):
            dt = sim.new_dt()
            sim.step(dt)
            dts.append(dt)
        P, U, B = sim.get_state()
        steps[case + "_prim0"] = prim
        steps[case + "_bfld0"] = bfld
        steps[case + "_dts"] = np.array(dts)
        steps[case + "_prim"] = P
        steps[case + "_cons"] = U
        steps[case + "_bfld"] = B
        steps[case + "_n"] = np.array([n_])
    np.savez_compressed(os.path.join(HERE, "steps.npz"), **steps)
    for f in ("kernels_mhd.npz", "kernels_hydro.npz", "steps.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)) // 1024, "KiB")


if __name__ == "__main__":
    main()
