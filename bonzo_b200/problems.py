"""Problem generators (initial conditions), seeded and host-side (numpy).

The reference binds one ``set_problem(grid, integr, usr_dir)`` per build
(src/problem/*.pyx, called at src/integration/vanleer.pyx:32); each writes the
primitive variables and the FACE-centred magnetic field on the active cells,
after which the integrator fills ghosts, interpolates the cell-centred field
from the faces and converts to conserved variables.  The generators here keep
that contract: they return ``(prim, bfld)`` arrays of shape (9, Nz, Ny, Nx) and
(3, Nz, Ny, Nx) over the full grid (ghosts left at zero) with the active
region and every face of every active cell set.

Magnetic fields are built from a vector potential sampled at cell edges and
differenced onto faces, so the discrete divergence vanishes to round-off.

All random inputs come from ``numpy.random.default_rng(seed)``.
"""
import math

import numpy as np

from .coords import GridCoord

RHO, VX, VY, VZ, PR, PSC, BX, BY, BZ = range(9)
NMODE = 9


def _empty(gc):
    return np.zeros((NMODE,) + gc.shape), np.zeros((3,) + gc.shape)


# ---------------------------------------------------------------------------
# Orszag-Tang vortex (src/problem/otvortex.pyx:42-66)
# ---------------------------------------------------------------------------

def otvortex(gc, beta=4 * math.pi, gam=5. / 3, pert_amp=0.0, pert_kmax=4, seed=0):
    """rho = gam^2, p = gam, v = (-sin 2 pi y, sin 2 pi x); B from the corner
    potential Az = cos(4 pi x)/(4 pi) + cos(2 pi y)/(2 pi), scaled by 1/sqrt(beta).

    With ``pert_amp`` > 0 a seeded smooth perturbation (Fourier modes with
    |k| <= pert_kmax, amplitude pert_amp) is added to vx, vy and Az.
    """
    if gc.dims != 2:
        raise ValueError("otvortex is a 2D problem")
    prim, bfld = _empty(gc)
    i1, i2, j1, j2 = gc.i1, gc.i2, gc.j1, gc.j2
    dx, dy = gc.dlf[0][i1], gc.dlf[1][j1]
    # corner potential on (j1..j2+1, i1..i2+1); corners at the left/bottom faces
    xc = gc.lv[0][i1:i2 + 2] - 0.5 * dx
    yc = gc.lv[1][j1:j2 + 2] - 0.5 * dy
    if i2 + 1 >= gc.Ntot[0]:
        raise ValueError("grid too small")
    Az = (np.cos(4 * math.pi * xc)[None, :] / (4 * math.pi)
          + np.cos(2 * math.pi * yc)[:, None] / (2 * math.pi))
    x = gc.lv[0][i1:i2 + 1]
    y = gc.lv[1][j1:j2 + 1]
    vx = np.broadcast_to(-np.sin(2 * math.pi * y)[:, None], (y.size, x.size)).copy()
    vy = np.broadcast_to(np.sin(2 * math.pi * x)[None, :], (y.size, x.size)).copy()
    if pert_amp > 0:
        rng = np.random.default_rng(seed)
        Lx, Ly = gc.Lglob[0], gc.Lglob[1]
        modes = [(kx, ky) for kx in range(-pert_kmax, pert_kmax + 1)
                 for ky in range(-pert_kmax, pert_kmax + 1)
                 if 0 < kx * kx + ky * ky <= pert_kmax * pert_kmax]

        def field(X, Y):
            out = np.zeros(np.broadcast(X, Y).shape)
            for (kx, ky) in modes:
                a, ph = rng.normal(), rng.uniform(0, 2 * math.pi)
                out += a * np.cos(2 * math.pi * (kx * X / Lx + ky * Y / Ly) + ph)
            return out / math.sqrt(len(modes))

        X, Y = np.meshgrid(x, y)
        vx += pert_amp * field(X, Y)
        vy += pert_amp * field(X, Y)
        Xc, Yc = np.meshgrid(xc, yc)
        Az = Az + pert_amp * field(Xc, Yc)
    a = gc.active
    prim[RHO][a] = gam * gam
    prim[PR][a] = gam
    prim[VX][a] = vx[None]
    prim[VY][a] = vy[None]
    sb = math.sqrt(beta)
    # faces i1..i2+1 (x) and j1..j2+1 (y) of every active cell
    bfld[0, 0, j1:j2 + 1, i1:i2 + 2] = (Az[1:, :] - Az[:-1, :]) / dy / sb + 1e-20
    bfld[1, 0, j1:j2 + 2, i1:i2 + 1] = -(Az[:, 1:] - Az[:, :-1]) / dx / sb + 1e-20
    return prim, bfld


# ---------------------------------------------------------------------------
# Blast wave (src/problem/blast_MHD.pyx:42-59), uneven-batch variant
# ---------------------------------------------------------------------------

def blast(gc, rho0=1.0, p0=0.1, b_mag=1.0 / math.sqrt(4 * math.pi), b_angle=math.pi / 4,
          center=(0.5, 0.5, 0.5), radius=0.1, p_ratio=100.0):
    """Uniform medium with an over-pressured sphere (disk in 2D) and a uniform
    field of magnitude b_mag at angle b_angle in the x-y plane."""
    prim, bfld = _empty(gc)
    a = gc.active
    x = gc.lv[0][gc.i1:gc.i2 + 1]
    y = gc.lv[1][gc.j1:gc.j2 + 1] if gc.dims >= 2 else np.array([0.0])
    z = gc.lv[2][gc.k1:gc.k2 + 1] if gc.dims >= 3 else np.array([0.0])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    L = gc.Lglob
    cx = center[0] * L[0]
    cy = center[1] * L[1] if gc.dims >= 2 else 0.0
    cz = center[2] * L[2] if gc.dims >= 3 else 0.0
    R = np.sqrt((X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2)
    prim[RHO][a] = rho0
    prim[PR][a] = np.where(R < radius, p0 * p_ratio, p0)
    bxv = b_mag * math.cos(b_angle)
    byv = b_mag * math.sin(b_angle)
    ks, js, is_ = a
    bfld[0][ks, js, gc.i1:gc.i2 + 2] = bxv
    if gc.dims >= 2:
        bfld[1][ks, gc.j1:gc.j2 + 2, is_] = byv
    else:
        bfld[1][a] = byv
    return prim, bfld


def blast_batch_params(n=64, seed=0, sizes=(64, 96, 128, 192, 256, 384, 512)):
    """Seeded draws for the uneven 2D blast sweep: per instance side length N,
    |B| = U(0.5, 2)/sqrt(4 pi) at angle U(0, 2 pi), disk centre U(0.2, 0.8)^2,
    pressure ratio U(10, 100)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(rng.choice(sizes))
        out.append(dict(N=N,
                        b_mag=float(rng.uniform(0.5, 2.0) / math.sqrt(4 * math.pi)),
                        b_angle=float(rng.uniform(0, 2 * math.pi)),
                        center=(float(rng.uniform(0.2, 0.8)), float(rng.uniform(0.2, 0.8)), 0.5),
                        p_ratio=float(rng.uniform(10, 100))))
    return out


# ---------------------------------------------------------------------------
# Periodic random fields (3D turbulence, conduction)
# ---------------------------------------------------------------------------

def _kgrid(N):
    k = [np.fft.fftfreq(n, 1.0 / n) for n in N]  # integer wavenumbers
    KZ, KY, KX = np.meshgrid(k[2], k[1], k[0], indexing="ij")
    return KX, KY, KZ


def _spectral_coeffs(N, rng, kmin, kmax, slope, ncomp):
    """Random complex coefficients with shell energy E(k) ~ k^slope on kmin<=|k|<=kmax."""
    KX, KY, KZ = _kgrid(N)
    K = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    mask = (K >= kmin) & (K <= kmax) & (K > 0)
    Ks = np.where(K > 0, K, 1.0)
    # 3D: E(k) ~ 4 pi k^2 |a(k)|^2  =>  |a| ~ k^((slope-2)/2)
    amp = np.where(mask, Ks ** ((slope - 2.0) / 2.0), 0.0)
    c = []
    for _ in range(ncomp):
        re = rng.normal(size=K.shape)
        im = rng.normal(size=K.shape)
        c.append(amp * (re + 1j * im))
    return c, (KX, KY, KZ)


def _eval(coef, kv, N, shift):
    """Real field sampled at cell offsets `shift` (in cells, per axis x,y,z)."""
    KX, KY, KZ = kv
    ph = np.exp(2j * math.pi * (KX * shift[0] / N[0] + KY * shift[1] / N[1] + KZ * shift[2] / N[2]))
    return np.real(np.fft.ifftn(coef * ph))


def _faces_from_edge_potential(gc, A):
    """Face B (3, Nz, Ny, Nx) from an edge vector potential on the periodic
    active block: A[0] on x-edges (cell-centre x, face y, face z) etc.
    B = curl A with the discrete Stokes theorem, so div B = 0 to round-off."""
    i1, j1, k1 = gc.i1, gc.j1, gc.k1
    Nx, Ny, Nz = gc.Nact
    dx, dy, dz = gc.dlf[0][i1], gc.dlf[1][j1], gc.dlf[2][k1]
    Ax, Ay, Az = A
    r = lambda F, ax: np.roll(F, -1, axis=ax)  # F at index+1 (periodic)
    # arrays are (z, y, x)
    bx = (r(Az, 1) - Az) / dy - (r(Ay, 0) - Ay) / dz
    by = (r(Ax, 0) - Ax) / dz - (r(Az, 2) - Az) / dx
    bz = (r(Ay, 2) - Ay) / dx - (r(Ax, 1) - Ax) / dy
    bf = np.zeros((3,) + gc.shape)
    ks, js, is_ = slice(k1, k1 + Nz), slice(j1, j1 + Ny), slice(i1, i1 + Nx)
    bf[0][ks, js, is_] = bx
    bf[1][ks, js, is_] = by
    bf[2][ks, js, is_] = bz
    # upper faces of the last active cells (periodic images of the first)
    bf[0][ks, js, i1 + Nx] = bx[:, :, 0]
    bf[1][ks, j1 + Ny, is_] = by[:, 0, :]
    bf[2][k1 + Nz, js, is_] = bz[0, :, :]
    return bf


def _random_potential(gc, rng, kmin, kmax, slope):
    N = gc.Nact
    c, kv = _spectral_coeffs(N, rng, kmin, kmax, slope, 3)
    # Ax on (x centre, y face, z face): shift (0, -1/2, -1/2) relative to centres
    Ax = _eval(c[0], kv, N, (0.0, -0.5, -0.5))
    Ay = _eval(c[1], kv, N, (-0.5, 0.0, -0.5))
    Az = _eval(c[2], kv, N, (-0.5, -0.5, 0.0))
    return (Ax, Ay, Az)


def turbulence3d(gc, seed=0, gam=5. / 3, rho0=1.0, p0=0.6, mach=1.0, beta=1.0,
                 kmin=2, kmax=16, slope=-5. / 3, b_pert=0.3):
    """Decaying MHD turbulence: solenoidal Gaussian velocity with E(k) ~ k^slope
    on kmin<=|k|<=kmax at rms Mach `mach`; B = B0 x-hat (beta = 2 p0 / B0^2) plus
    the curl of a random edge potential with the same spectrum at b_pert*B0 rms."""
    if gc.dims != 3:
        raise ValueError("turbulence3d is a 3D problem")
    rng = np.random.default_rng(seed)
    N = gc.Nact
    c, (KX, KY, KZ) = _spectral_coeffs(N, rng, kmin, kmax, slope, 3)
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    K2s = np.where(K2 > 0, K2, 1.0)
    kdotc = (KX * c[0] + KY * c[1] + KZ * c[2]) / K2s
    c = [c[0] - KX * kdotc, c[1] - KY * kdotc, c[2] - KZ * kdotc]
    v = [np.real(np.fft.ifftn(ci)) for ci in c]
    cs = math.sqrt(gam * p0 / rho0)
    vrms = math.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    v = [vi * (mach * cs / vrms) for vi in v]
    prim, _ = _empty(gc)
    a = gc.active
    prim[RHO][a] = rho0
    prim[PR][a] = p0
    prim[VX][a], prim[VY][a], prim[VZ][a] = v
    B0 = math.sqrt(2.0 * p0 / beta)
    A = _random_potential(gc, rng, kmin, kmax, slope)
    bf = _faces_from_edge_potential(gc, A)
    brms = math.sqrt(np.mean(bf[0][a] ** 2 + bf[1][a] ** 2 + bf[2][a] ** 2))
    bf *= b_pert * B0 / brms
    i1, Nx = gc.i1, gc.Nact[0]
    bf[0][a[0], a[1], i1:i1 + Nx + 1] += B0
    return prim, bf


def conduction3d(gc, seed=0, rho0=1.0, t_amp=0.5, kmax=8, slope=-2.0, beta=100.0,
                 b_pert=0.1, t_floor=0.2):
    """rho = 1, T = max(1 + t_amp G, t_floor) (G Gaussian, E(k) ~ k^slope on
    |k|<=kmax, unit rms), p = rho T; B = B0 x-hat with beta = 2<p>/B0^2 plus b_pert*B0 rms random-A field."""
    if gc.dims != 3:
        raise ValueError("conduction3d is a 3D problem")
    rng = np.random.default_rng(seed)
    N = gc.Nact
    c, kv = _spectral_coeffs(N, rng, 1, kmax, slope, 1)
    G = np.real(np.fft.ifftn(c[0]))
    G /= math.sqrt(np.mean(G ** 2))
    # positivity: a unit-rms Gaussian reaches -4..-5 on large grids, so the
    # temperature is floored at t_floor (a clip of the far tail)
    T = np.maximum(1.0 + t_amp * G, t_floor)
    prim, _ = _empty(gc)
    a = gc.active
    prim[RHO][a] = rho0
    prim[PR][a] = rho0 * T
    B0 = math.sqrt(2.0 * float(np.mean(rho0 * T)) / beta)
    A = _random_potential(gc, rng, 1, kmax, slope)
    bf = _faces_from_edge_potential(gc, A)
    brms = math.sqrt(np.mean(bf[0][a] ** 2 + bf[1][a] ** 2 + bf[2][a] ** 2))
    bf *= b_pert * B0 / brms
    i1, Nx = gc.i1, gc.Nact[0]
    bf[0][a[0], a[1], i1:i1 + Nx + 1] += B0
    return prim, bf


# ---------------------------------------------------------------------------
# Known-answer problems
# ---------------------------------------------------------------------------

def thcond_gauss(gc, sig=0.15, bx=0.1):
    """src/problem/thcond_gauss.pyx:35-52: rho = 1, p = exp(-r^2/sig^2) + 1
    centred in the box, Bx = bx (run with gam = 2)."""
    prim, bfld = _empty(gc)
    a = gc.active
    L = gc.Lglob
    x = gc.lv[0][gc.i1:gc.i2 + 1]
    y = gc.lv[1][gc.j1:gc.j2 + 1] if gc.dims >= 2 else np.array([0.0])
    z = gc.lv[2][gc.k1:gc.k2 + 1] if gc.dims >= 3 else np.array([0.0])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r2 = (X - 0.5 * L[0]) ** 2
    if gc.dims >= 2:
        r2 = r2 + (Y - 0.5 * L[1]) ** 2
    if gc.dims >= 3:
        r2 = r2 + (Z - 0.5 * L[2]) ** 2
    prim[RHO][a] = 1.0
    prim[PR][a] = np.exp(-r2 / sig ** 2) + 1.0
    bfld[0][a[0], a[1], gc.i1:gc.i2 + 2] = bx
    return prim, bfld


def linear_wave(gc, wave="fast", amp=1e-6, gam=5. / 3, rho0=1.0, p0=1.0 / (5. / 3),
                b0=(1.0, math.sqrt(2.0), 0.5), kdir=(1, 0, 0)):
    """Small-amplitude MHD eigenmode along x (after linwaves2d.pyx:84-190):
    right-going fast / Alfven / slow / entropy wave with amplitude `amp`,
    background rho0, p0, B = b0 (Bx along the propagation direction)."""
    if kdir != (1, 0, 0):
        raise ValueError("only x-propagating waves are generated")
    prim, bfld = _empty(gc)
    a = gc.active
    Bx, By, Bz = b0
    L = gc.Lglob[0]
    x = gc.lv[0][gc.i1:gc.i2 + 1]
    # eigenvector in primitive variables of the 1D MHD system along x
    a2 = gam * p0 / rho0
    ca2 = Bx * Bx / rho0
    bt2 = (By * By + Bz * Bz) / rho0
    cf2 = 0.5 * (a2 + ca2 + bt2 + math.sqrt((a2 + ca2 + bt2) ** 2 - 4 * a2 * ca2))
    cs2 = 0.5 * (a2 + ca2 + bt2 - math.sqrt((a2 + ca2 + bt2) ** 2 - 4 * a2 * ca2))
    bt = math.sqrt(By * By + Bz * Bz)
    by_, bz_ = (By / bt, Bz / bt) if bt > 0 else (1.0 / math.sqrt(2), 1.0 / math.sqrt(2))
    sgn = 1.0 if Bx >= 0 else -1.0
    if wave in ("fast", "slow"):
        c2 = cf2 if wave == "fast" else cs2
        c = math.sqrt(c2)
        # d rho, d vx, d vy, d vz, d p, d By, d Bz per unit d rho
        # linearised 1D MHD along x with d rho = 1: d vx = c/rho, d p = a^2,
        # d Bt = c^2 Bt / (rho (c^2 - ca^2)), d vt = -Bx c Bt / (rho^2 (c^2 - ca^2))
        dvx = c / rho0
        dvt = -Bx * c / (rho0 * (c2 - ca2)) * (bt / rho0) if (c2 - ca2) != 0 else 0.0
        dbt = c2 / (c2 - ca2) * bt / rho0 if (c2 - ca2) != 0 else 0.0
        ev = dict(rho=1.0, vx=dvx, vy=dvt * by_, vz=dvt * bz_, p=a2, by=dbt * by_, bz=dbt * bz_)
        speed = c
    elif wave == "alfven":
        ev = dict(rho=0.0, vx=0.0, vy=-bz_, vz=by_, p=0.0,
                  by=sgn * bz_ * math.sqrt(rho0), bz=-sgn * by_ * math.sqrt(rho0))
        speed = math.sqrt(ca2)
    elif wave == "entropy":
        ev = dict(rho=1.0, vx=0.0, vy=0.0, vz=0.0, p=0.0, by=0.0, bz=0.0)
        speed = 0.0
    else:
        raise ValueError(wave)
    s = np.sin(2 * math.pi * x / L)
    prim[RHO][a] = rho0 + amp * ev["rho"] * s
    prim[VX][a] = amp * ev["vx"] * s
    prim[VY][a] = amp * ev["vy"] * s
    prim[VZ][a] = amp * ev["vz"] * s
    prim[PR][a] = p0 + amp * ev["p"] * s
    ks, js, is_ = a
    bfld[0][ks, js, gc.i1:gc.i2 + 2] = Bx
    bfld[1][a] = By + amp * ev["by"] * s
    bfld[2][a] = Bz + amp * ev["bz"] * s
    if gc.dims >= 2:
        bfld[1][ks, gc.j2 + 1, is_] = bfld[1][ks, gc.j1, is_]
    if gc.dims >= 3:
        bfld[2][gc.k2 + 1, js, is_] = bfld[2][gc.k1, js, is_]
    return prim, bfld, speed


def make_grid(Nx, Ny=1, Nz=1, dims=2, bc=0, reconstr="linear", lmin=(0., 0., 0.),
              lmax=(1., 1., 1.)):
    """Convenience: GridCoord with one BC flag on every side (or a 3x2 table)."""
    if isinstance(bc, int):
        bc = ((bc, bc), (bc, bc), (bc, bc))
    ng = 2 if reconstr == "const" else 3
    return GridCoord(Nx, Ny, Nz, dims, lmin, lmax, bc, ng)


# ---------------------------------------------------------------------------
# set_problem(grid, integr, usr_dir) entry points for bonzo_b200.Simulation:
# parameters from the [problem] section (read_user_param), as the reference's
# src/problem/*.pyx read them; each fills grid.prim and grid.bfld.
# ---------------------------------------------------------------------------

def _fill(grid, prim, bfld):
    grid.prim[...] = prim
    grid.bfld[...] = bfld


def _user(usr_dir, key, dtype, default):
    from .config import read_user_param
    return read_user_param(key, dtype, usr_dir, default)


def set_problem_otvortex(grid, integr, usr_dir):
    """src/problem/otvortex.pyx: beta from [problem] beta (default 4 pi);
    optional seeded perturbation: pert_amp, pert_kmax, seed."""
    prim, bfld = otvortex(grid.coord, beta=_user(usr_dir, "beta", "f", 4 * math.pi), gam=integr.gam,
                          pert_amp=_user(usr_dir, "pert_amp", "f", 0.0),
                          pert_kmax=_user(usr_dir, "pert_kmax", "i", 4), seed=_user(usr_dir, "seed", "i", 0))
    _fill(grid, prim, bfld)


def set_problem_blast(grid, integr, usr_dir):
    """src/problem/blast_MHD.pyx: rho = 1, p = 10 inside r < 0.1 of the box
    centre and 0.1 outside, B = (1, 1, 1) / sqrt(1.5 beta) ([problem] beta);
    the uneven-batch parameters (b_mag, b_angle, p_ratio, center) override."""
    gc = grid.coord
    beta = _user(usr_dir, "beta", "f", 1.0)
    bt = 1.0 / math.sqrt(1.5 * beta)
    prim, bfld = blast(gc, rho0=1.0, p0=0.1, b_mag=_user(usr_dir, "b_mag", "f", bt * math.sqrt(2.0)),
                       b_angle=_user(usr_dir, "b_angle", "f", math.pi / 4),
                       center=(_user(usr_dir, "xc", "f", 0.5), _user(usr_dir, "yc", "f", 0.5),
                               _user(usr_dir, "zc", "f", 0.5)),
                       radius=_user(usr_dir, "radius", "f", 0.1), p_ratio=_user(usr_dir, "p_ratio", "f", 100.0))
    # the reference's blast also carries Bz = bt (cell-centred face in 2D)
    a = gc.active
    ks, js, is_ = a
    if gc.dims >= 3:
        bfld[2][gc.k1:gc.k2 + 2, js, is_] = _user(usr_dir, "bz", "f", bt)
    else:
        bfld[2][a] = _user(usr_dir, "bz", "f", bt)
    _fill(grid, prim, bfld)


def set_problem_turbulence3d(grid, integr, usr_dir):
    """Decaying driven-free MHD turbulence (seed, mach, beta, kmax from [problem])."""
    prim, bfld = turbulence3d(grid.coord, seed=_user(usr_dir, "seed", "i", 0), gam=integr.gam,
                              mach=_user(usr_dir, "mach", "f", 1.0), beta=_user(usr_dir, "beta", "f", 1.0),
                              kmax=_user(usr_dir, "kmax", "i", 16))
    _fill(grid, prim, bfld)


def set_problem_conduction3d(grid, integr, usr_dir):
    """Field-aligned conduction test box (seed, kmax, beta from [problem])."""
    prim, bfld = conduction3d(grid.coord, seed=_user(usr_dir, "seed", "i", 0), kmax=_user(usr_dir, "kmax", "i", 8),
                              beta=_user(usr_dir, "beta", "f", 100.0))
    _fill(grid, prim, bfld)


def set_problem_thcond_gauss(grid, integr, usr_dir):
    """src/problem/thcond_gauss.pyx: Gaussian temperature profile along B."""
    prim, bfld = thcond_gauss(grid.coord, sig=_user(usr_dir, "sig", "f", 0.15), bx=_user(usr_dir, "bx", "f", 0.1))
    _fill(grid, prim, bfld)


def set_problem_linear_wave(grid, integr, usr_dir):
    """Linear MHD eigenmode (src/problem/linwaves2d.pyx): wave fast/alfven/slow/entropy, amp."""
    prim, bfld, _ = linear_wave(grid.coord, _user(usr_dir, "wave", "s", "fast"), amp=_user(usr_dir, "amp", "f", 1e-6),
                                gam=integr.gam)
    _fill(grid, prim, bfld)


SET_PROBLEM = {
    "otvortex": set_problem_otvortex,
    "blast": set_problem_blast,
    "turbulence3d": set_problem_turbulence3d,
    "conduction3d": set_problem_conduction3d,
    "thcond_gauss": set_problem_thcond_gauss,
    "linear_wave": set_problem_linear_wave,
}
