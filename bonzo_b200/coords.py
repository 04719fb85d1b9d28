"""Grid indices and Cartesian coordinates (host side, numpy).

Follows the reference's index and coordinate conventions exactly:
  - ghost width ng = 3 for linear and 2 for constant reconstruction
    (src/coordinates/grid.pyx:127-134);
  - active cells i1..i2 = ng..Nx+ng-1, and Ntot = Nx + 2 ng on active axes,
    Ntot = 1 on inactive ones (grid.pyx:140-160);
  - face coordinates lf[i] = l1 + (i - i1) dx with dx = (lmax - lmin)/Nact and
    ghost faces rebuilt from the periodic / reflected active spacings
    (src/coordinates/coord.pyx:189-246);
  - lv = (lf[i] + lf[i+1])/2, dlf = lf[i+1] - lf[i], dlv = lv[i] - lv[i-1]
    and their inverses (coord.pyx:251-256, src/coordinates/cartesian.pyx:18-43).
The same arithmetic runs in the C++ context (bonzo_b200/csrc/bnz_ctx.cu), so
the device kernels see bit-identical spacings.
"""
import numpy as np

BC_PERIODIC, BC_OUTFLOW, BC_REFLECT = 0, 1, 2


class GridCoord:
    def __init__(self, Nx, Ny=1, Nz=1, dims=2, lmin=(0., 0., 0.), lmax=(1., 1., 1.),
                 bc=((0, 0), (0, 0), (0, 0)), ng=3):
        if dims not in (1, 2, 3):
            raise ValueError("dims must be 1, 2 or 3")
        self.dims = dims
        self.ng = ng
        Na = [int(Nx), int(Ny) if dims >= 2 else 1, int(Nz) if dims >= 3 else 1]
        if dims < 2 and int(Ny) != 1:
            raise ValueError("cannot set Ny>1 without second dimension")
        if dims < 3 and int(Nz) != 1:
            raise ValueError("cannot set Nz>1 without third dimension")
        self.Nact = Na
        self.Ntot = [Na[a] + 2 * ng if a < dims else 1 for a in range(3)]
        self.i1, self.i2 = ng, Na[0] + ng - 1
        self.j1, self.j2 = (ng, Na[1] + ng - 1) if dims >= 2 else (0, 0)
        self.k1, self.k2 = (ng, Na[2] + ng - 1) if dims >= 3 else (0, 0)
        self.lmin = [float(v) for v in lmin]
        self.lmax = [float(v) for v in lmax]
        self.bc = [tuple(int(f) for f in b) for b in bc]
        self.lf, self.lv, self.dlf, self.dlf_inv, self.dlv, self.dlv_inv = [], [], [], [], [], []
        for n in range(3):
            self._axis(n)

    def _axis(self, n):
        Ntot = self.Ntot[n]
        lf = np.zeros(Ntot + 1)
        if Ntot == 1:
            lf[0], lf[1] = self.lmin[n], self.lmax[n]
        else:
            ind1 = (self.i1, self.j1, self.k1)[n]
            ind2 = (self.i2, self.j2, self.k2)[n]
            dx = (self.lmax[n] - self.lmin[n]) / self.Nact[n]
            l1 = 0 * self.Nact[n] * dx  # pos = 0 without MPI
            for i in range(Ntot + 1):
                lf[i] = l1 + (i - ind1) * dx
            b0, b1 = self.bc[n]
            if b0 == BC_PERIODIC:
                for i in range(ind1 - 1, -1, -1):
                    i_ = ind2 - i + (ind1 - 1)
                    lf[i] = lf[i + 1] - (lf[i_ + 1] - lf[i_])
            if b1 == BC_PERIODIC:
                for i in range(ind2 + 1, Ntot):
                    i_ = ind1 + i - (ind2 + 1)
                    lf[i + 1] = lf[i] + (lf[i_ + 1] - lf[i_])
            if b0 == BC_REFLECT:
                for i in range(ind1 - 1, -1, -1):
                    i_ = ind1 - i + (ind1 - 1)
                    lf[i] = lf[i + 1] - (lf[i_ + 1] - lf[i_])
            if b1 == BC_REFLECT:
                for i in range(ind2 + 1, Ntot):
                    i_ = ind2 - i + (ind2 + 1)
                    lf[i + 1] = lf[i] + (lf[i_ + 1] - lf[i_])
        dlf = lf[1:] - lf[:-1]
        dlf_inv = 1.0 / dlf
        lv = 0.5 * (lf[:-1] + lf[1:])
        dlv = np.zeros(Ntot)
        dlv_inv = np.zeros(Ntot)
        if Ntot > 1:
            dlv[1:] = lv[1:] - lv[:-1]
            dlv_inv[1:] = 1.0 / dlv[1:]
        self.lf.append(lf)
        self.lv.append(lv)
        self.dlf.append(dlf)
        self.dlf_inv.append(dlf_inv)
        self.dlv.append(dlv)
        self.dlv_inv.append(dlv_inv)

    @property
    def shape(self):
        """(Nz_tot, Ny_tot, Nx_tot): the trailing shape of prim / cons / bfld."""
        return (self.Ntot[2], self.Ntot[1], self.Ntot[0])

    @property
    def active(self):
        """Slices of the active region in (k, j, i) order."""
        return (slice(self.k1, self.k2 + 1), slice(self.j1, self.j2 + 1),
                slice(self.i1, self.i2 + 1))

    @property
    def Lglob(self):
        return [self.lmax[n] - self.lmin[n] for n in range(3)]
