"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker or the timed CPU reference.  The shipped
library (bonzo_b200) never imports it.

Two native libraries stand behind it:
  oracle/_build/libbnzoracle*.so  the C restatement (oracle/bnz_oracle.c)
  oracle/_ref/libbnzref*.so       the reference's own C kernels, compiled from
                                  its sources by oracle/build_ref.py when the
                                  reference tree is present (optional).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NMODE = 9
NVAR = 12
RS = {"hll": 0, "hllc": 1, "hlld": 2, "hllt": 3}
RCN = {"const": 0, "linear": 1}
LIM = {"vl": 0, "mc": 1, "mm": 2}
TC = {"iso": 0, "aniso": 1}

_dp = C.POINTER(C.c_double)


class OrcParams(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("dims", C.c_int),
        ("lmin", C.c_double * 3), ("lmax", C.c_double * 3),
        ("bc", (C.c_int * 2) * 3),
        ("gam", C.c_double), ("cour", C.c_double),
        ("rsolver", C.c_int), ("reconstr", C.c_int), ("limiter", C.c_int),
        ("charact_proj", C.c_int),
        ("kappa0", C.c_double), ("thcond_type", C.c_int), ("sat_hfe", C.c_int),
        ("cour_diff", C.c_double),
        ("fixdt", C.c_int), ("dt_fixed", C.c_double),
        ("outflow_face_aware", C.c_int),
        ("nthreads", C.c_int), ("rows_parallel", C.c_int),
        ("grav", C.c_double * 3), ("drive_f0", C.c_double), ("drive_tau", C.c_double),
        ("drive_nmod", C.c_int), ("drive_seed", C.c_uint64),
    ]


_libs = {}


def _lib(hydro=False):
    key = "hydro" if hydro else "mhd"
    if key not in _libs:
        name = "libbnzoracle_hydro.so" if hydro else "libbnzoracle.so"
        path = os.path.join(HERE, "_build", name)
        if not os.path.exists(path):
            raise RuntimeError("oracle library %s missing: run oracle/build.py" % path)
        L = C.CDLL(path)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [C.c_void_p]
        for f in ("orc_ntot",):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int]
            getattr(L, f).restype = C.c_int
        L.orc_ng.argtypes = [C.c_void_p]
        L.orc_ng.restype = C.c_int
        L.orc_get_coord.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        L.orc_set_kernels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_set_state.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_init.argtypes = [C.c_void_p]
        L.orc_new_dt.argtypes = [C.c_void_p]
        L.orc_new_dt.restype = C.c_double
        L.orc_vl2_step.argtypes = [C.c_void_p, C.c_double]
        L.orc_diffuse.argtypes = [C.c_void_p, C.c_double]
        L.orc_apply_bc.argtypes = [C.c_void_p, C.c_uint32]
        L.orc_advance.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.orc_time.argtypes = [C.c_void_p]
        L.orc_time.restype = C.c_double
        L.orc_step_count.argtypes = [C.c_void_p]
        L.orc_step_count.restype = C.c_long
        L.orc_last_dt.argtypes = [C.c_void_p]
        L.orc_last_dt.restype = C.c_double
        L.orc_last_nsts.argtypes = [C.c_void_p]
        L.orc_last_nsts.restype = C.c_int
        L.orc_flux_flat.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_int, C.c_double]
        L.orc_reconstr_flat.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int,
                                        C.c_double]
        L.orc_fms.argtypes = [_dp, C.c_double, C.c_double]
        L.orc_fms.restype = C.c_double
        L.orc_coord_block.argtypes = [C.c_void_p]
        L.orc_coord_block.restype = C.c_void_p
        L.orc_reconstr_flat_with.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int,
                                             C.c_double, C.c_void_p]
        L.orc_get_nsts.argtypes = [C.c_double, C.c_double]
        L.orc_get_nsts.restype = C.c_int
        L.orc_get_sts_coeff.argtypes = [C.c_int, _dp]
        _libs[key] = L
    return _libs[key]


def _ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def ref_lib(hydro=False):
    """The reference's compiled kernels, or None when oracle/_ref was not built."""
    name = "libbnzref_hydro.so" if hydro else "libbnzref.so"
    path = os.path.join(HERE, "_ref", name)
    if not os.path.exists(path):
        return None
    key = "ref_" + name
    if key not in _libs:
        _libs[key] = C.CDLL(path)
    return _libs[key]


def _rows(a):
    """real** over the rows of a 2-D C-contiguous float64 array."""
    n = a.shape[0]
    arr = (_dp * n)()
    for m in range(n):
        arr[m] = a[m].ctypes.data_as(_dp)
    return arr


def ref_row_eos(name, a, gam, hydro=False):
    """The reference's cons2prim_1 / prim2cons_1 over a flat (NMODE, n) array."""
    L = ref_lib(hydro)
    if L is None:
        raise RuntimeError("oracle/_ref not built")
    fn = getattr(L, name)
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double]
    a = np.ascontiguousarray(a)
    out = np.zeros_like(a)
    fn(_rows(out), _rows(a), 0, a.shape[1] - 1, gam)
    return out


def orc_row_eos(name, a, gam, hydro=False):
    L = _lib(hydro)
    fn = getattr(L, "orc_" + name)
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double]
    a = np.ascontiguousarray(a)
    out = np.zeros_like(a)
    fn(_rows(out), _rows(a), 0, a.shape[1] - 1, gam)
    return out


def ref_fms(w, gam, hydro=False):
    L = ref_lib(hydro)
    if L is None:
        raise RuntimeError("oracle/_ref not built")
    L.fms.argtypes = [_dp, C.c_double, C.c_double]
    L.fms.restype = C.c_double
    w = np.ascontiguousarray(w, dtype=np.float64)
    return L.fms(_ptr(w), 0.0, gam)


def ref_flux_flat(rsolver, wl, wr, bx, gam, hydro=False):
    """Call the reference's own hll/hllc/hllt/hlld_flux over flat arrays (NMODE, n)."""
    L = ref_lib(hydro)
    if L is None:
        raise RuntimeError("oracle/_ref not built")
    fn = getattr(L, rsolver + "_flux")
    nm, n = wl.shape
    flux = np.zeros((nm, n))
    wl = np.ascontiguousarray(wl)
    wr = np.ascontiguousarray(wr)
    bx = np.ascontiguousarray(bx)
    fn.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int, C.c_double]
    fn(_rows(flux), _rows(wl), _rows(wr), bx.ctypes.data_as(_dp), 0, n - 1, gam)
    return flux


def orc_flux_flat(rsolver, wl, wr, bx, gam, hydro=False):
    L = _lib(hydro)
    nm, n = wl.shape
    flux = np.zeros((nm, n))
    L.orc_flux_flat(RS[rsolver], _ptr(flux), _ptr(np.ascontiguousarray(wl)),
                    _ptr(np.ascontiguousarray(wr)), _ptr(np.ascontiguousarray(bx)), n, gam)
    return flux


def orc_reconstr_flat(reconstr, limiter, w, gam, char_proj=0, hydro=False):
    """Reconstruct one row w (NMODE, n): returns wl, wr (NMODE, n+1), cells 1..n-2."""
    L = _lib(hydro)
    nm, n = w.shape
    wl = np.zeros((nm, n + 1))
    wr = np.zeros((nm, n + 1))
    L.orc_reconstr_flat(RCN[reconstr], LIM[limiter], char_proj, _ptr(wl), _ptr(wr),
                        _ptr(np.ascontiguousarray(w)), n, gam)
    return wl, wr


def reconstr_with(fn_name, order, w, gam, use_ref=False, hydro=False, char_proj=0):
    """Run the reference's (use_ref) or the restated reconstruction function
    `fn_name` ('reconstr_const' / 'reconstr_linear') on one row w (NMODE, n)."""
    L = _lib(hydro)
    nm, n = w.shape
    wl = np.zeros((nm, n + 1))
    wr = np.zeros((nm, n + 1))
    if use_ref:
        R = ref_lib(hydro)
        if R is None:
            raise RuntimeError("oracle/_ref not built")
        fn = C.cast(getattr(R, fn_name), C.c_void_p)
    else:
        fn = C.cast(getattr(L, "orc_" + fn_name), C.c_void_p)
    sim = OracleSim(Nx=max(n, 8), Ny=1, Nz=1, dims=1, hydro=hydro)
    L.orc_reconstr_flat_with(fn, order, char_proj, _ptr(wl), _ptr(wr), _ptr(np.ascontiguousarray(w)),
                             n, gam, L.orc_coord_block(sim.h))
    del sim
    return wl, wr


def orc_fms(w, gam, hydro=False):
    w = np.ascontiguousarray(w, dtype=np.float64)
    return _lib(hydro).orc_fms(_ptr(w), 0.0, gam)


def get_sts_coeff(s):
    c = np.zeros((s + 1) * 4)
    _lib().orc_get_sts_coeff(s, _ptr(c))
    return c.reshape(s + 1, 4)


def get_nsts(dt_hyp, dt_diff):
    return _lib().orc_get_nsts(dt_hyp, dt_diff)


class OracleSim:
    """One grid advanced by the oracle (vanleer.advance restated in C)."""

    def __init__(self, Nx, Ny=1, Nz=1, dims=2, lmin=(0., 0., 0.), lmax=(1., 1., 1.),
                 bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4, rsolver="hlld",
                 reconstr="linear", limiter="vl", charact_proj=0, kappa0=0.,
                 thcond_type="aniso", sat_hfe=0, cour_diff=0.5, fixdt=False, dt_fixed=0.,
                 outflow_face_aware=1, nthreads=0, rows_parallel=1, use_ref_kernels=False,
                 hydro=False, grav=(0., 0., 0.), drive_f0=0., drive_tau=1., drive_nmod=1, drive_seed=0):
        self.hydro = hydro
        self.L = _lib(hydro)
        p = OrcParams()
        p.Nx, p.Ny, p.Nz, p.dims = Nx, Ny, Nz, dims
        for a in range(3):
            p.lmin[a] = lmin[a]
            p.lmax[a] = lmax[a]
            p.bc[a][0] = bc[a][0]
            p.bc[a][1] = bc[a][1]
        p.gam, p.cour = gam, cour
        p.rsolver, p.reconstr, p.limiter = RS[rsolver], RCN[reconstr], LIM[limiter]
        p.charact_proj = charact_proj
        p.kappa0, p.thcond_type, p.sat_hfe, p.cour_diff = kappa0, TC[thcond_type], sat_hfe, cour_diff
        p.fixdt, p.dt_fixed = int(bool(fixdt)), dt_fixed
        p.outflow_face_aware = outflow_face_aware
        p.nthreads, p.rows_parallel = nthreads, rows_parallel
        for a in range(3):
            p.grav[a] = grav[a]
        p.drive_f0, p.drive_tau, p.drive_nmod, p.drive_seed = drive_f0, drive_tau, drive_nmod, drive_seed
        self.params = p
        self.h = self.L.orc_create(C.byref(p))
        self.nmode = 6 if hydro else NMODE
        self.shape = (self.L.orc_ntot(self.h, 2), self.L.orc_ntot(self.h, 1),
                      self.L.orc_ntot(self.h, 0))
        self.ng = self.L.orc_ng(self.h)
        self.dims = dims
        self._keep = []
        if use_ref_kernels:
            R = ref_lib(hydro)
            if R is None:
                raise RuntimeError("oracle/_ref not built")
            rs = C.cast(getattr(R, rsolver + "_flux"), C.c_void_p)
            rc0 = C.cast(R.reconstr_const, C.c_void_p)
            rc1 = C.cast(R.reconstr_linear, C.c_void_p) if limiter == "vl" else None
            self.L.orc_set_kernels(self.h, rs, rc0, rc1)

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass

    def coords(self, ax):
        N = self.L.orc_ntot(self.h, ax)
        lf = np.zeros(N + 1)
        lv = np.zeros(N)
        dlf = np.zeros(N)
        self.L.orc_get_coord(self.h, ax, _ptr(lf), _ptr(lv), _ptr(dlf))
        return lf, lv, dlf

    def set_state(self, prim, bfld=None):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        assert prim.shape == (self.nmode,) + self.shape
        bp = None
        if bfld is not None:
            bfld = np.ascontiguousarray(bfld, dtype=np.float64)
            assert bfld.shape == (3,) + self.shape
            bp = _ptr(bfld)
        self.L.orc_set_state(self.h, _ptr(prim), bp)

    def init(self):
        self.L.orc_init(self.h)

    def get_state(self):
        prim = np.zeros((self.nmode,) + self.shape)
        cons = np.zeros((self.nmode,) + self.shape)
        bfld = np.zeros((3,) + self.shape)
        self.L.orc_get_state(self.h, _ptr(prim), _ptr(cons), _ptr(bfld))
        return prim, cons, bfld

    def new_dt(self):
        return self.L.orc_new_dt(self.h)

    def step(self, dt):
        self.L.orc_vl2_step(self.h, dt)

    def apply_bc(self, mask=(1 << NVAR) - 1):
        self.L.orc_apply_bc(self.h, mask)

    def advance(self, tmax, max_steps=0):
        self.L.orc_advance(self.h, tmax, max_steps)

    @property
    def time(self):
        return self.L.orc_time(self.h)

    @property
    def nstep(self):
        return self.L.orc_step_count(self.h)

    @property
    def last_dt(self):
        return self.L.orc_last_dt(self.h)

    @property
    def last_nsts(self):
        return self.L.orc_last_nsts(self.h)
