"""FP64 torch transcription of one 2D VL2 step (PLM + HLL/HLLD + CT) with the
boundary index maps of the fused device path.  Test infrastructure only: a
slow, differentiable second implementation that the tests compare with the
oracle (forward) and with the hand-written adjoint (torch autograd).

It restates, in vectorised torch, the same algorithm as oracle/bnz_oracle.c:
the predictor of src/integration/vanleer.pyx:104-120 (donor cell, dt/2, cells
1..Ntot-2), the corrector of vanleer.pyx:130-151 (PLM, dt, active cells), the
Riemann solvers of src/mhd/fluxes_c.c:175-223 (HLL), :447-607 (HLLT) and
:616-834 (HLLD), the limiters of src/coordinates/reconstr_c.h:28-44 (with the
characteristic projection of reconstr_c.c:54-91 and src/mhd/eos_c.h:100-333
as an option), constant gravity (src/srcterms/gravity.pyx:54-69) and the CT
update of src/integration/ct.pyx:15-215.  Ghost values are read through the boundary
maps of src/bc/grid_bc_funcs.pyx (periodic, outflow with the face-aware
option, reflect), as the fused path does.

State layout: prim (9, ny, nx), bfld (3, ny, nx) -- the (9 | 3, 1, Ny, Nx)
arrays of the library with the z axis dropped.
"""
import numpy as np
import torch

RHO, VX, VY, VZ, PR, PSC, BX, BY, BZ = range(9)
PERM_Y = [RHO, VY, VZ, VX, PR, PSC, BY, BZ, BX]  # local n -> global variable (y sweep)


class Branches:
    """Records every branch decision of the step (limiter cases, Riemann fan
    regions, min / max of wave speeds, signs under |x|) and replays them: with
    the decisions frozen the step is a smooth function of its inputs, so
    central differences of it converge to the derivative at the recording point
    (the branch-frozen check of a discrete adjoint)."""

    def __init__(self):
        self.mode = None
        self.masks = []
        self.pos = 0

    def record(self):
        self.mode, self.masks, self.pos = "record", [], 0

    def replay(self):
        self.mode, self.pos = "replay", 0

    def off(self):
        self.mode = None


BRANCHES = Branches()


def cond(mask):
    """A branch decision: recorded, replayed or passed through."""
    b = BRANCHES
    if b.mode == "record":
        b.masks.append(mask)
    elif b.mode == "replay":
        mask = b.masks[b.pos]
        b.pos += 1
    return mask


def branch_sign(x):
    return torch.where(cond(x > 0), torch.ones_like(x), torch.where(cond(x < 0), -torch.ones_like(x),
                                                                      torch.zeros_like(x)))


# ---------------------------------------------------------------------------
# boundary index maps (the fused path's map_cell / map_face)
# ---------------------------------------------------------------------------

def axis_maps(ntot, ng, n, f0, f1, face_aware):
    a1, a2 = ng, ng + n - 1
    cs, cf = np.arange(ntot), np.zeros(ntot, bool)
    fs, ff, fz = np.arange(ntot), np.zeros(ntot, bool), np.zeros(ntot, bool)
    for a in range(ntot):
        if a < a1:
            cs[a], cf[a] = (a + n, False) if f0 == 0 else (a1, False) if f0 == 1 else (2 * a1 - 1 - a, True)
            fs[a], ff[a] = (a + n, False) if f0 == 0 else (a1, False) if f0 == 1 else (2 * a1 - a, True)
        elif a > a2:
            cs[a], cf[a] = (a - n, False) if f1 == 0 else (a2, False) if f1 == 1 else (2 * a2 + 1 - a, True)
            if f1 == 0:
                fs[a] = a - n
            elif f1 == 1:
                fs[a] = (a if a == a2 + 1 else a2 + 1) if face_aware else a2
            elif a == a2 + 1:
                fz[a] = True
            else:
                fs[a], ff[a] = 2 * a2 + 2 - a, True
        if a == a1 and f0 == 2:
            fz[a] = True
    return cs, cf, fs, ff, fz


class Grid:
    """Index maps and coordinates of a 2D grid (bonzo_b200.coords.GridCoord)."""

    def __init__(self, gc, face_aware=True, device="cpu"):
        self.ng = gc.ng
        self.nx, self.ny = gc.Ntot[0], gc.Ntot[1]
        self.N = gc.Nact[:2]
        self.R1 = (gc.i1, gc.i2, gc.j1, gc.j2)
        self.R0 = (1, self.nx - 2, 1, self.ny - 2)
        t = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64, device=device)
        self.lf = [t(gc.lf[a]) for a in range(2)]
        self.lv = [t(gc.lv[a]) for a in range(2)]
        self.dlf = [t(gc.dlf[a]) for a in range(2)]
        self.dlf_inv = [t(gc.dlf_inv[a]) for a in range(2)]
        self.dz = float(gc.dlf[2][0])
        mx = axis_maps(self.nx, self.ng, self.N[0], gc.bc[0][0], gc.bc[0][1], face_aware)
        my = axis_maps(self.ny, self.ng, self.N[1], gc.bc[1][0], gc.bc[1][1], face_aware)
        li = lambda a: torch.as_tensor(a, dtype=torch.long, device=device)
        sg = lambda f: torch.as_tensor(np.where(f, -1.0, 1.0), dtype=torch.float64, device=device)
        self.cx, self.cy = li(mx[0]), li(my[0])
        self.cx_s, self.cy_s = sg(mx[1]), sg(my[1])
        self.fx, self.fy = li(mx[2]), li(my[2])
        self.fx_s = sg(mx[3]) * torch.as_tensor(~mx[4], dtype=torch.float64, device=device)
        self.fy_s = sg(my[3]) * torch.as_tensor(~my[4], dtype=torch.float64, device=device)

    def read_cells(self, w):
        """w as the step reads it: ghost cells through the maps (with flips)."""
        r = w[:, self.cy][:, :, self.cx]
        sx = self.cx_s[None, :]
        sy = self.cy_s[:, None]
        out = [r[v] for v in range(9)]
        out[VX], out[BX] = out[VX] * sx, out[BX] * sx
        out[VY], out[BY] = out[VY] * sy, out[BY] * sy
        return torch.stack(out)

    def read_faces(self, b):
        bx = b[0][self.cy][:, self.fx] * self.fx_s[None, :]
        by = b[1][self.fy][:, self.cx] * self.fy_s[:, None]
        bz = b[2][self.cy][:, self.cx]
        return torch.stack([bx, by, bz])


# ---------------------------------------------------------------------------
# per-point math (lists of 9 tensors, local sweep frame)
# ---------------------------------------------------------------------------

def prim2cons(w, gam):
    v2 = w[VX] ** 2 + w[VY] ** 2 + w[VZ] ** 2
    b2 = w[BX] ** 2 + w[BY] ** 2 + w[BZ] ** 2
    return [w[RHO], w[RHO] * w[VX], w[RHO] * w[VY], w[RHO] * w[VZ],
            0.5 * (w[RHO] * v2 + b2) + w[PR] / (gam - 1.0), w[PSC], w[BX], w[BY], w[BZ]]


def cons2prim(u, gam):
    rhoi = 1.0 / u[RHO]
    vx, vy, vz = u[1] * rhoi, u[2] * rhoi, u[3] * rhoi
    v2 = vx ** 2 + vy ** 2 + vz ** 2
    b2 = u[BX] ** 2 + u[BY] ** 2 + u[BZ] ** 2
    p = (gam - 1.0) * (u[4] - 0.5 * (b2 + v2 * u[RHO]))
    return [u[RHO], vx, vy, vz, p, u[PSC], u[BX], u[BY], u[BZ]]


def flux(w, u):
    bx2 = w[BX] ** 2
    b2 = bx2 + w[BY] ** 2 + w[BZ] ** 2
    pt = 0.5 * b2 + w[PR]
    f = [u[n] * w[VX] for n in range(6)]
    f[1] = f[1] + pt - bx2
    f[2] = f[2] - w[BX] * w[BY]
    f[3] = f[3] - w[BX] * w[BZ]
    f[4] = f[4] + pt * w[VX] - (w[VX] * bx2 + w[VY] * w[BX] * w[BY] + w[VZ] * w[BX] * w[BZ])
    zero = torch.zeros_like(w[RHO])
    return f + [zero, w[VX] * w[BY] - w[VY] * w[BX], w[VX] * w[BZ] - w[VZ] * w[BX]]


def fms(w, gam):
    bx2 = w[BX] ** 2
    b2 = bx2 + w[BY] ** 2 + w[BZ] ** 2
    gamp = gam * w[PR]
    c1 = gamp + b2
    disc = c1 * c1 - 4.0 * gamp * bx2
    c2 = torch.sqrt(torch.where(cond(disc >= 0), disc, -disc))
    return torch.sqrt(0.5 / w[RHO] * (c1 + c2))


def wave_speeds(wL, wR, gam):
    # fmin / fmax with the first argument taken on ties, which is also the
    # branch the device adjoint differentiates (torch.minimum would split the
    # gradient of a tie between both arguments)
    cfL, cfR = fms(wL, gam), fms(wR, gam)
    cf = torch.where(cond(cfL >= cfR), cfL, cfR)
    vmin = torch.where(cond(wL[VX] <= wR[VX]), wL[VX], wR[VX])
    vmax = torch.where(cond(wL[VX] >= wR[VX]), wL[VX], wR[VX])
    return vmin - cf, vmax + cf


def hll(wL, wR, gam):
    uL, uR = prim2cons(wL, gam), prim2cons(wR, gam)
    fL, fR = flux(wL, uL), flux(wR, uR)
    sL, sR = wave_speeds(wL, wR, gam)
    aL = torch.where(cond(sL < 0), sL, torch.zeros_like(sL))
    aR = torch.where(cond(sR > 0), sR, torch.zeros_like(sR))
    inv = 1.0 / (aR - aL)
    out = [(aR * fL[n] - aL * fR[n] + aL * aR * (uR[n] - uL[n])) * inv for n in range(9)]
    out[BX] = torch.zeros_like(out[0])
    return out


def hlld(wL, wR, gam):
    bx = wL[BX]
    bx2 = bx ** 2
    sL, sR = wave_speeds(wL, wR, gam)
    uL, uR = prim2cons(wL, gam), prim2cons(wR, gam)
    fL, fR = flux(wL, uL), flux(wR, uR)
    ptL = wL[PR] + 0.5 * (bx2 + wL[BY] ** 2 + wL[BZ] ** 2)
    ptR = wR[PR] + 0.5 * (bx2 + wR[BY] ** 2 + wR[BZ] ** 2)
    deni = 1.0 / (sR * uR[RHO] - sL * uL[RHO] - (fR[RHO] - fL[RHO]))
    sM = (sR * uR[1] - sL * uL[1] - (fR[1] - fL[1])) * deni
    star = {}
    for side, w, u, s, pt in (("L", wL, uL, sL, ptL), ("R", wR, uR, sR, ptR)):
        svx = s - w[VX]
        sMi = 1.0 / (s - sM)
        x = svx * sMi
        rs = w[RHO] * x
        rv = w[RHO] * svx
        wvb = 1.0 / (rv * (s - sM) - bx2)
        wv = bx * (sM - w[VX]) * wvb
        vys = w[VY] - w[BY] * wv
        vzs = w[VZ] - w[BZ] * wv
        wb = (rv * svx - bx2) * wvb
        bys, bzs = w[BY] * wb, w[BZ] * wb
        vsbs = sM * bx + vys * bys + vzs * bzs
        star[side] = dict(svx=svx, sMi=sMi, x=x, rs=rs, vys=vys, vzs=vzs, bys=bys, bzs=bzs, vsbs=vsbs,
                          sr=torch.sqrt(rs), pt=pt)
    pts = wL[RHO] * star["L"]["svx"] * (sM - wL[VX]) + ptL
    sgnb = branch_sign(bx)
    absbx = sgnb * bx
    sLs = sM - absbx / star["L"]["sr"]
    sRs = sM + absbx / star["R"]["sr"]
    srL, srR = star["L"]["sr"], star["R"]["sr"]
    rhoLRi = 1.0 / (srL + srR)
    L_, R_ = star["L"], star["R"]
    vyss = (srL * L_["vys"] + srR * R_["vys"] + (R_["bys"] - L_["bys"]) * sgnb) * rhoLRi
    vzss = (srL * L_["vzs"] + srR * R_["vzs"] + (R_["bzs"] - L_["bzs"]) * sgnb) * rhoLRi
    byss = (srL * R_["bys"] + srR * L_["bys"] + srL * srR * (R_["vys"] - L_["vys"]) * sgnb) * rhoLRi
    bzss = (srL * R_["bzs"] + srR * L_["bzs"] + srL * srR * (R_["vzs"] - L_["vzs"]) * sgnb) * rhoLRi
    vssbss = sM * bx + vyss * byss + vzss * bzss
    res = {}
    for side, w, u, f, s, si, sign in (("L", wL, uL, fL, sL, sLs, -1.0), ("R", wR, uR, fR, sR, sRs, 1.0)):
        q = star[side]
        dot = w[VX] * bx + w[VY] * w[BY] + w[VZ] * w[BZ]
        es = (q["svx"] * u[4] - q["pt"] * w[VX] + pts * sM + bx * (dot - q["vsbs"])) * q["sMi"]
        zero = torch.zeros_like(es)
        us = [q["rs"], q["rs"] * sM, q["rs"] * q["vys"], q["rs"] * q["vzs"], es, u[PSC] * q["x"], zero,
              q["bys"], q["bzs"]]
        t = q["sr"] * (q["vsbs"] - vssbss) * sgnb
        ess = es + sign * t
        uss = [q["rs"], q["rs"] * sM, q["rs"] * vyss, q["rs"] * vzss, ess, u[PSC] * q["x"], zero, byss, bzss]
        res[side] = (f, [f[n] + s * (us[n] - u[n]) for n in range(9)],
                     [f[n] + s * (us[n] - u[n]) + si * (uss[n] - us[n]) for n in range(9)])
    r1 = cond(sL > 0)
    r2 = cond((sL <= 0) & (0 < sLs))
    r3 = cond((sLs <= 0) & (0 < sM))
    r4 = cond((sM <= 0) & (0 < sRs))
    r5 = cond((sRs <= 0) & (0 < sR))
    r6 = cond(sR <= 0)
    out = []
    for n in range(9):
        # the reference's sequential tests: the last true one wins
        v = torch.zeros_like(sM)
        for m, val in ((r1, res["L"][0][n]), (r2, res["L"][1][n]), (r3, res["L"][2][n]),
                       (r4, res["R"][2][n]), (r5, res["R"][1][n]), (r6, res["R"][0][n])):
            v = torch.where(m, val, v)
        out.append(v)
    out[BX] = torch.zeros_like(out[0])
    return out


def hllt(wL, wR, gam):
    """The three-wave solver of fluxes_c.c:447-607 as the device restates it
    (bnz_device.cuh flux_hllt): star-state energies zero, a zero flux where no
    fan region matches."""
    uL, uR = prim2cons(wL, gam), prim2cons(wR, gam)
    fL, fR = flux(wL, uL), flux(wR, uR)
    sL, sR = wave_speeds(wL, wR, gam)
    bx = wL[BX]
    sRsLi = 1.0 / (sR - sL)
    rhos = (sR * uR[RHO] - sL * uL[RHO] - (fR[RHO] - fL[RHO])) * sRsLi
    mxs = (sR * uR[1] - sL * uL[1] - (fR[1] - fL[1])) * sRsLi
    frhos = (sR * fL[RHO] - sL * fR[RHO] + sR * sL * (uR[RHO] - uL[RHO])) * sRsLi
    us = frhos / rhos
    pscs = (sR * uR[PSC] - sL * uL[PSC] - (fR[PSC] - fL[PSC])) * sRsLi
    rhosi = 1.0 / rhos
    sqri = torch.sqrt(rhosi)
    sgnb = branch_sign(bx)
    absbx = sgnb * bx
    sLs = us - absbx * sqri
    sRs = us + absbx * sqri
    zero = torch.zeros_like(rhos)
    star = {}
    for side, w, s in (("L", wL, sL), ("R", wR, sR)):
        xs = 1.0 / ((s - sLs) * (s - sRs))
        y1 = bx * xs * (us - w[VX])
        y2 = (w[RHO] * (s - w[VX]) ** 2 - bx ** 2) * rhosi * xs
        star[side] = [rhos, mxs, rhos * w[VY] - y1 * w[BY], rhos * w[VZ] - y1 * w[BZ], zero, pscs, zero,
                      y2 * w[BY], y2 * w[BZ]]
    uLs, uRs = star["L"], star["R"]
    x = 0.5 * sgnb / sqri
    uCs = [rhos, mxs,
           0.5 * (uLs[VY] + uRs[VY]) + x * (uRs[BY] - uLs[BY]),
           0.5 * (uLs[VZ] + uRs[VZ]) + x * (uRs[BZ] - uLs[BZ]),
           zero, pscs, zero,
           0.5 * (uLs[BY] + uRs[BY]) + x * rhosi * (uRs[VY] - uLs[VY]),
           0.5 * (uLs[BZ] + uRs[BZ]) + x * rhosi * (uRs[VZ] - uLs[VZ])]
    r1 = cond(sL > 0)
    r2 = cond((sL <= 0) & (0 < sLs))
    r3 = cond((sLs <= 0) & (0 < sRs))
    r4 = cond((sRs <= 0) & (0 < sR))
    r5 = cond(sR <= 0)
    out = []
    for n in range(9):
        lstar = fL[n] + sL * (uLs[n] - uL[n])
        v = torch.zeros_like(rhos)
        for m, val in ((r1, fL[n]), (r2, lstar), (r3, lstar + sLs * (uCs[n] - uLs[n])),
                       (r4, fR[n] + sR * (uRs[n] - uR[n])), (r5, fR[n])):
            v = torch.where(m, val, v)
        out.append(v)
    out[BX] = torch.zeros_like(out[0])
    return out


def _abs(x):
    return torch.where(cond(x >= 0), x, -x)


def _char_basis(w, gam):
    """The eigen-system coefficients that prim2char / char2prim of
    src/mhd/eos_c.h:100-216, 245-333 (bnz_device.cuh) build from the cell
    state w (local sweep frame)."""
    rho, p, bx, by, bz = w[RHO], w[PR], w[BX], w[BY], w[BZ]
    rhoi = 1.0 / rho
    s = branch_sign(bx)
    a2rho = gam * p
    a = torch.sqrt(a2rho * rhoi)
    bx2 = bx ** 2
    bperp2 = by ** 2 + bz ** 2
    x = a2rho + (bx2 + bperp2)
    y = torch.sqrt(_abs(x * x - 4.0 * a2rho * bx2))
    cf2rho = 0.5 * (x + y)
    cs2rho = 0.5 * (x - y)
    cf = torch.sqrt(rhoi * cf2rho)
    cs = torch.sqrt(rhoi * _abs(cs2rho))
    z = 1.0 / (cf2rho - cs2rho)
    one, zero = torch.ones_like(rho), torch.zeros_like(rho)
    c1, c2, c3 = cond(cf <= cs), cond(a <= cs), cond(cf <= a)
    af = torch.where(c1, one, torch.where(c2, zero, torch.where(c3, one, torch.sqrt(z * _abs(a2rho - cs2rho)))))
    as_ = torch.where(c1, zero, torch.where(c2, one, torch.where(c3, zero, torch.sqrt(z * _abs(cf2rho - a2rho)))))
    nz = cond(bperp2 != 0)
    bperpi = 1.0 / torch.sqrt(torch.where(nz, bperp2, one))
    betay = torch.where(nz, bperpi * by, zero)
    betaz = torch.where(nz, bperpi * bz, zero)
    return dict(rho=rho, rhoi=rhoi, s=s, a2rho=a2rho, a=a, cf=cf, cs=cs, af=af, as_=as_, betay=betay, betaz=betaz)


def prim2char(d, k):
    """Differences d (9, local frame) into the characteristic basis; PSC and
    BX pass through."""
    rhoi, s, a, cf, cs = k["rhoi"], k["s"], k["a"], k["cf"], k["cs"]
    by_, bz_ = k["betay"], k["betaz"]
    nf = 0.5 / (k["a2rho"] * rhoi)
    qf_ = nf * cf * k["af"] * s
    qs_ = nf * cs * k["as_"] * s
    af_ = nf * k["af"]
    as__ = nf * k["as_"]
    rhoisr = torch.sqrt(rhoi)
    arhoisr = a * rhoisr
    Af_ = af_ * arhoisr
    As_ = as__ * arhoisr
    x = s * rhoisr
    v = by_ * d[VY] + bz_ * d[VZ]
    b = by_ * d[BY] + bz_ * d[BZ]
    out = list(d)
    out[RHO] = af_ * (rhoi * d[PR] - cf * d[VX]) + qs_ * v + As_ * b
    out[VX] = 0.5 * ((-bz_ * d[VY] + by_ * d[VZ]) + x * (-bz_ * d[BY] + by_ * d[BZ]))
    out[VY] = as__ * (rhoi * d[PR] - cs * d[VX]) - qf_ * v - Af_ * b
    out[VZ] = d[RHO] - 2.0 * nf * d[PR]
    out[PR] = as__ * (rhoi * d[PR] + cs * d[VX]) + qf_ * v - Af_ * b
    out[BY] = 0.5 * ((bz_ * d[VY] - by_ * d[VZ]) + x * (-bz_ * d[BY] + by_ * d[BZ]))
    out[BZ] = af_ * (rhoi * d[PR] + cf * d[VX]) - qs_ * v + As_ * b
    return out


def char2prim(c, k):
    """Characteristic amplitudes c (9) back to primitive differences."""
    rho, s, a, cf, cs, af, as_ = k["rho"], k["s"], k["a"], k["cf"], k["cs"], k["af"], k["as_"]
    by_, bz_ = k["betay"], k["betaz"]
    qf = cf * af * s
    qs = cs * as_ * s
    rhosr = torch.sqrt(rho)
    arhosr = a * rhosr
    Af = af * arhosr
    As = as_ * arhosr
    fa = af * (c[RHO] + c[BZ]) + as_ * (c[VY] + c[PR])
    t = qs * (c[RHO] - c[BZ]) - qf * (c[VY] - c[PR])
    u = As * (c[RHO] + c[BZ]) - Af * (c[VY] + c[PR])
    out = list(c)
    out[RHO] = rho * fa + c[VZ]
    out[VX] = cf * af * (c[BZ] - c[RHO]) + cs * as_ * (c[PR] - c[VY])
    out[VY] = by_ * t - bz_ * (c[VX] - c[BY])
    out[VZ] = bz_ * t + by_ * (c[VX] - c[BY])
    out[PR] = k["a2rho"] * fa
    out[BY] = by_ * u - bz_ * s * rhosr * (c[VX] + c[BY])
    out[BZ] = bz_ * u + by_ * s * rhosr * (c[VX] + c[BY])
    return out


def half_slopes_char(wm, wc, wp, gam, lim):
    """reconstr_c.c:54-91 with charact_proj: the one-sided differences of all
    nine local variables projected on the cell's characteristic basis,
    limited, halved and projected back."""
    k = _char_basis(wc, gam)
    dm = prim2char([wc[n] - wm[n] for n in range(9)], k)
    dp = prim2char([wp[n] - wc[n] for n in range(9)], k)
    return char2prim([0.5 * limit(lim, dm[n], dp[n]) for n in range(9)], k)


def _mm(a, b):
    return torch.where(cond(a * b <= 0), torch.zeros_like(a),
                       torch.where(cond(a > 0), torch.where(cond(a < b), a, b), torch.where(cond(a > b), a, b)))


def limit(lim, a, b):
    if lim == "mm":
        return _mm(a, b)
    if lim == "mc":
        return _mm(2.0 * _mm(a, b), 0.5 * (a + b))
    ab = a * b
    pos = cond(ab > 0)
    s = torch.where(pos, a + b, torch.ones_like(a))
    return torch.where(pos, 2.0 * ab / s, torch.zeros_like(a))


# ---------------------------------------------------------------------------
# one stage of the step and the whole step
# ---------------------------------------------------------------------------

def _plm_faces(c, gam, lim, charact):
    """Face states from the four cells c[0..3] (local frame) around each face:
    wL from the slope of c[1], wR from that of c[2]."""
    if charact:
        dL = half_slopes_char(c[0], c[1], c[2], gam, lim)
        dR = half_slopes_char(c[1], c[2], c[3], gam, lim)
        return [c[1][v] + dL[v] for v in range(9)], [c[2][v] - dR[v] for v in range(9)]
    wL = [c[1][v] + 0.5 * limit(lim, c[1][v] - c[0][v], c[2][v] - c[1][v]) for v in range(9)]
    wR = [c[2][v] - 0.5 * limit(lim, c[2][v] - c[1][v], c[3][v] - c[2][v]) for v in range(9)]
    return wL, wR


def stage(G, Wf, Bf, Wn, Bn, dt, order, R, gam, rs, lim, grav=None, charact=False):
    """Fluxes, EMFs and the update on cells R = (ia, ib, ja, jb).  Wf / Bf are
    the cell / face arrays the fluxes read, Wn / Bn the state whose u^n and
    faces are updated (all as read).  With `grav` (gx, gy, gz) the constant
    gravity source of src/srcterms/gravity.pyx:54-69 is added after the update,
    with the density and velocity of the stage input Wf.  Returns prim (9, R),
    bx faces (R rows, ia..ib+1), by faces (ja..jb+1, R columns), bz (R)."""
    ia, ib, ja, jb = R
    solver = {"hlld": hlld, "hllt": hllt}.get(rs, hll)
    # x faces i = ia..ib+1 on rows ja-1..jb+1
    rows = slice(ja - 1, jb + 2)
    if order == 0:
        wL = [Wf[v][rows, ia - 1:ib + 1] for v in range(9)]
        wR = [Wf[v][rows, ia:ib + 2] for v in range(9)]
    else:
        c = [[Wf[v][rows, ia - 2 + q:ib + q] for v in range(9)] for q in range(4)]
        wL, wR = _plm_faces(c, gam, lim, charact)
    wL[BX] = wR[BX] = Bf[0][rows, ia:ib + 2]
    Fx = solver(wL, wR, gam)                      # (jb-ja+3, ib-ia+2), global order
    # y faces j = ja..jb+1 on columns ia-1..ib+1
    cols = slice(ia - 1, ib + 2)
    if order == 0:
        wL = [Wf[PERM_Y[n]][ja - 1:jb + 1, cols] for n in range(9)]
        wR = [Wf[PERM_Y[n]][ja:jb + 2, cols] for n in range(9)]
    else:
        c = [[Wf[PERM_Y[n]][ja - 2 + q:jb + q, cols] for n in range(9)] for q in range(4)]
        wL, wR = _plm_faces(c, gam, lim, charact)
    wL[BX] = wR[BX] = Bf[1][ja:jb + 2, cols]
    fy = solver(wL, wR, gam)
    Fy = [None] * 9
    for n in range(9):
        Fy[PERM_Y[n]] = fy[n]                     # (jb-ja+2, ib-ia+3)
    # cell-centred E_z on cells ia-1..ib+1, ja-1..jb+1 and corner E_z
    ec = -(Wf[VX][ja - 1:jb + 2, ia - 1:ib + 2] * Wf[BY][ja - 1:jb + 2, ia - 1:ib + 2] -
           Wf[VY][ja - 1:jb + 2, ia - 1:ib + 2] * Wf[BX][ja - 1:jb + 2, ia - 1:ib + 2])
    # corners (ia..ib+1, ja..jb+1): Fx[BY] at x faces rows cj-1, cj; Fy[BX] at y faces cols ci-1, ci
    fxby = Fx[BY]
    fybx = Fy[BX]
    E = (0.5 * (-fxby[0:-1, :] - fxby[1:, :] + fybx[:, 0:-1] + fybx[:, 1:]) -
         0.25 * (ec[1:, 0:-1] + ec[1:, 1:] + ec[0:-1, 0:-1] + ec[0:-1, 1:]))
    # update
    dx = G.dlf[0][ia:ib + 1][None, :]
    dy = G.dlf[1][ja:jb + 1][:, None]
    dz = G.dz
    vol = dx * dy * dz
    dtdv = dt / vol
    dax = dy * dz
    day = dx * dz
    wn = [Wn[v][ja:jb + 1, ia:ib + 1] for v in range(9)]
    un = prim2cons(wn, gam)
    u = [None] * 9
    for n in range(6):
        v = un[n] - dtdv * (dax * Fx[n][1:-1, 1:] - dax * Fx[n][1:-1, :-1])
        u[n] = v - dtdv * (day * Fy[n][1:, 1:-1] - day * Fy[n][:-1, 1:-1])
    # faces
    dyf = G.dlf[1][ja:jb + 1][:, None]
    dtda = dt / (dyf * dz)
    bxf = Bn[0][ja:jb + 1, ia:ib + 2] - dtda * (dz * E[1:, :] - dz * E[:-1, :])
    dxf = G.dlf[0][ia:ib + 1][None, :]
    dtda = dt / (dxf * dz)
    byf = Bn[1][ja:jb + 2, ia:ib + 1] + dtda * (dz * E[:, 1:] - dz * E[:, :-1])
    dtda = dt / (dx * dy)
    eyl, eyr = Fx[BZ][1:-1, :-1], Fx[BZ][1:-1, 1:]
    exb, ext = -Fy[BZ][:-1, 1:-1], -Fy[BZ][1:, 1:-1]
    bz = Bn[2][ja:jb + 1, ia:ib + 1] - dtda * (dy * eyr - dy * eyl)
    bz = bz + dtda * (dx * ext - dx * exb)
    lvx, lfx, dix = G.lv[0][ia:ib + 1], G.lf[0], G.dlf_inv[0][ia:ib + 1]
    lvy, lfy, diy = G.lv[1][ja:jb + 1], G.lf[1], G.dlf_inv[1][ja:jb + 1]
    u[BX] = ((lvx - lfx[ia:ib + 1])[None, :] * bxf[:, :-1] + (lfx[ia + 1:ib + 2] - lvx)[None, :] * bxf[:, 1:]) * \
        dix[None, :]
    u[BY] = ((lvy - lfy[ja:jb + 1])[:, None] * byf[:-1, :] + (lfy[ja + 1:jb + 2] - lvy)[:, None] * byf[1:, :]) * \
        diy[:, None]
    u[BZ] = bz
    if grav is not None:
        rho, vx, vy, vz = (Wf[v][ja:jb + 1, ia:ib + 1] for v in (RHO, VX, VY, VZ))
        u[VX] = u[VX] + rho * grav[0] * dt
        u[VY] = u[VY] + rho * grav[1] * dt
        u[VZ] = u[VZ] + rho * grav[2] * dt
        u[PR] = u[PR] + dt * ((rho * vx) * grav[0] + (rho * vy) * grav[1] + (rho * vz) * grav[2])
    return torch.stack(cons2prim(u, gam)), bxf, byf, bz


def step(G, prim, bfld, dt, gam=5.0 / 3.0, rs="hlld", lim="vl", grav=None, charact=False):
    """One VL2 step: returns (prim, bfld) as the library's get_state gives them
    (ghosts filled through the maps).  `grav`: constant gravity (gx, gy, gz),
    none when absent or all zero."""
    if grav is not None and not any(g != 0.0 for g in grav):
        grav = None
    wr = G.read_cells(prim)
    br = G.read_faces(bfld)
    ia, ib, ja, jb = G.R0
    ws_, bxs, bys, bzs = stage(G, wr, br, wr, br, 0.5 * dt, 0, G.R0, gam, rs, lim, grav)
    Ws = torch.zeros_like(prim)
    Ws[:, ja:jb + 1, ia:ib + 1] = ws_
    Bs = torch.zeros_like(bfld)
    Bs[0, ja:jb + 1, ia:ib + 2] = bxs
    Bs[1, ja:jb + 2, ia:ib + 1] = bys
    Bs[2, ja:jb + 1, ia:ib + 1] = bzs
    ia, ib, ja, jb = G.R1
    w1, bx1, by1, bz1 = stage(G, Ws, Bs, wr, br, dt, 1, G.R1, gam, rs, lim, grav, charact)
    C = torch.zeros_like(prim)
    C[:, ja:jb + 1, ia:ib + 1] = w1
    Cb = torch.zeros_like(bfld)
    Cb[0, ja:jb + 1, ia:ib + 2] = bx1
    Cb[1, ja:jb + 2, ia:ib + 1] = by1
    Cb[2, ja:jb + 1, ia:ib + 1] = bz1
    return G.read_cells(C), G.read_faces(Cb)
