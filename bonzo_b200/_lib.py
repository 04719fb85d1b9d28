"""ctypes binding of libbnzgpu.so (the C ABI in include/bnz_gpu.h).

The library is built in-tree by bonzo_b200/build.py.  There is no CPU
fallback: if the shared library is missing, or no CUDA device is visible, the
calls fail loudly with BnzError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbnzgpu.so")

BNZ_OK, BNZ_ERR_ARG, BNZ_ERR_CUDA, BNZ_ERR_STATE, BNZ_ERR_UNSUPPORTED, BNZ_ERR_TIMEOUT, BNZ_ERR_NOMEM = range(7)
STATUS_NAMES = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "non-physical state",
                4: "unsupported", 5: "timeout", 6: "out of memory"}
RS = {"hll": 0, "hllc": 1, "hlld": 2, "hllt": 3}
RCN = {"const": 0, "linear": 1}
LIM = {"vl": 0, "mc": 1, "mm": 2}
TC = {"iso": 0, "aniso": 1}
PATH = {"fused": 0, "plain": 1, "split": 2}

# every entry point include/bnz_gpu.h declares (checked by the CPU tests)
EXPORTS = [
    "bnz_create", "bnz_destroy", "bnz_last_error", "bnz_shape", "bnz_set_state", "bnz_init",
    "bnz_get_state", "bnz_apply_bc", "bnz_new_dt", "bnz_vl2_step", "bnz_diffuse", "bnz_advance",
    "bnz_get_time", "bnz_last_nsts", "bnz_set_time", "bnz_check", "bnz_sync", "bnz_advance_graph",
    "bnz_device_state", "bnz_stream", "bnz_set_stream", "bnz_launch_count",
    "bnz_batch_create", "bnz_batch_destroy", "bnz_batch_last_error", "bnz_batch_size",
    "bnz_batch_instance", "bnz_batch_advance", "bnz_batch_advance_timed", "bnz_batch_step_host", "bnz_batch_test_withhold_loads", "bnz_fp64_fma_peak", "bnz_fast_rcp", "bnz_batch_set_stream", "bnz_batch_launch_count",
    "bnz_batch_sync", "bnz_variant_count", "bnz_batch_set_variant", "bnz_batch_get_variant",
    "bnz_batch_time_variant", "bnz_batch_autotune", "bnz_vl2_step_noalloc", "bnz_noalloc_last_error",
    "bnz_noalloc_check", "bnz_noalloc_scratch_bytes", "bnz_set_state_device", "bnz_get_state_device", "bnz_rollout_forward",
    "bnz_rollout_adjoint", "bnz_step_adjoint", "bnz_history", "bnz_div_b", "bnz_riemann", "bnz_snapshot", "bnz_snapshot_wait",
]


class BnzError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS_NAMES.get(code, "error"), code, msg))
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("dims", C.c_int),
                ("lmin", C.c_double * 3), ("lmax", C.c_double * 3), ("bc", (C.c_int * 2) * 3)]


class MethodDesc(C.Structure):
    _fields_ = [("gam", C.c_double), ("cour", C.c_double),
                ("rsolver", C.c_int), ("reconstr", C.c_int), ("limiter", C.c_int),
                ("charact_proj", C.c_int),
                ("kappa0", C.c_double), ("thcond_type", C.c_int), ("sat_hfe", C.c_int),
                ("cour_diff", C.c_double), ("fixdt", C.c_int), ("dt_fixed", C.c_double),
                ("outflow_face_aware", C.c_int), ("exact_fp", C.c_int), ("path", C.c_int),
                ("grav", C.c_double * 3), ("drive_f0", C.c_double), ("drive_tau", C.c_double),
                ("drive_nmod", C.c_int), ("drive_seed", C.c_uint64), ("hydro", C.c_int)]


_dp = C.POINTER(C.c_double)
_lib = None


def load():
    """Load libbnzgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BnzError(BNZ_ERR_UNSUPPORTED, "libbnzgpu.so not built: run bonzo_b200/build.py "
                       "(no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.bnz_create.argtypes = [C.POINTER(GridDesc), C.POINTER(MethodDesc), C.POINTER(vp)]
    L.bnz_destroy.argtypes = [vp]
    L.bnz_last_error.argtypes = [vp]
    L.bnz_last_error.restype = C.c_char_p
    L.bnz_shape.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.bnz_set_state.argtypes = [vp, _dp, C.c_int, _dp]
    L.bnz_init.argtypes = [vp]
    L.bnz_get_state.argtypes = [vp, _dp, _dp, _dp]
    L.bnz_apply_bc.argtypes = [vp, C.c_uint32]
    L.bnz_new_dt.argtypes = [vp, _dp]
    L.bnz_vl2_step.argtypes = [vp, C.c_double]
    L.bnz_diffuse.argtypes = [vp, C.c_double, C.POINTER(C.c_int)]
    L.bnz_advance.argtypes = [vp, C.c_double, C.c_int, _dp, C.POINTER(C.c_long)]
    L.bnz_get_time.argtypes = [vp, _dp, C.POINTER(C.c_long), _dp]
    L.bnz_set_time.argtypes = [vp, C.c_double, C.c_long]
    L.bnz_last_nsts.argtypes = [vp, C.POINTER(C.c_int)]
    L.bnz_check.argtypes = [vp, C.POINTER(C.c_uint32)]
    L.bnz_sync.argtypes = [vp]
    L.bnz_advance_graph.argtypes = [vp, C.c_double, C.c_int]
    L.bnz_device_state.argtypes = [vp, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp)]
    L.bnz_stream.argtypes = [vp, C.POINTER(vp)]
    L.bnz_set_stream.argtypes = [vp, vp]
    L.bnz_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.bnz_batch_create.argtypes = [C.POINTER(GridDesc), C.c_int, C.POINTER(MethodDesc), C.POINTER(vp)]
    L.bnz_batch_destroy.argtypes = [vp]
    L.bnz_batch_last_error.argtypes = [vp]
    L.bnz_batch_last_error.restype = C.c_char_p
    L.bnz_batch_size.argtypes = [vp, C.POINTER(C.c_int)]
    L.bnz_batch_instance.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.bnz_batch_advance.argtypes = [vp, C.c_double, C.c_int]
    L.bnz_batch_advance_timed.argtypes = [vp, C.c_double, C.c_int, _dp]
    L.bnz_fp64_fma_peak.argtypes = [_dp]
    L.bnz_fast_rcp.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.bnz_batch_test_withhold_loads.argtypes = [vp, C.c_int]
    L.bnz_batch_step_host.argtypes = [vp, C.POINTER(_dp), C.POINTER(_dp), C.c_double, C.c_int, C.c_int]
    L.bnz_set_state_device.argtypes = [vp, vp, vp]
    L.bnz_get_state_device.argtypes = [vp, vp, vp]
    L.bnz_rollout_forward.argtypes = [vp, C.c_int, C.c_double, C.c_int]
    L.bnz_rollout_adjoint.argtypes = [vp, vp, vp, vp, vp]
    L.bnz_step_adjoint.argtypes = [vp, C.c_double, vp, vp, vp, vp, vp, vp]
    L.bnz_history.argtypes = [vp, _dp]
    L.bnz_div_b.argtypes = [vp, _dp]
    L.bnz_riemann.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_int, C.c_double, C.c_int, vp, vp]
    L.bnz_snapshot.argtypes = [vp, _dp, _dp, _dp]
    L.bnz_snapshot_wait.argtypes = [vp]
    L.bnz_batch_set_stream.argtypes = [vp, vp]
    L.bnz_batch_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.bnz_batch_sync.argtypes = [vp]
    ip = C.POINTER(C.c_int)
    L.bnz_variant_count.argtypes = [ip, ip, ip, ip, ip]
    L.bnz_batch_set_variant.argtypes = [vp, C.c_int]
    L.bnz_batch_get_variant.argtypes = [vp, ip]
    L.bnz_batch_time_variant.argtypes = [vp, C.c_int, C.c_int, _dp]
    L.bnz_batch_autotune.argtypes = [vp, C.c_int, ip, _dp]
    _lib = L
    return L


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 C-contiguous array expected"
    return a.ctypes.data_as(_dp)


def grid_desc(Nx, Ny=1, Nz=1, dims=2, lmin=(0., 0., 0.), lmax=(1., 1., 1.),
              bc=((0, 0), (0, 0), (0, 0))):
    g = GridDesc()
    g.Nx, g.Ny, g.Nz, g.dims = Nx, Ny, Nz, dims
    for a in range(3):
        g.lmin[a], g.lmax[a] = lmin[a], lmax[a]
        g.bc[a][0], g.bc[a][1] = bc[a][0], bc[a][1]
    return g


def method_desc(gam=5. / 3, cour=0.4, rsolver="hlld", reconstr="linear", limiter="vl",
                charact_proj=0, kappa0=0.0, thcond_type="aniso", sat_hfe=0, cour_diff=0.5,
                fixdt=False, dt_fixed=0.0, outflow_face_aware=1, exact_fp=False, path="plain",
                grav=(0.0, 0.0, 0.0), drive_f0=0.0, drive_tau=1.0, drive_nmod=1, drive_seed=0, hydro=False):
    m = MethodDesc()
    m.gam, m.cour = gam, cour
    m.rsolver = RS[rsolver] if isinstance(rsolver, str) else rsolver
    m.reconstr = RCN[reconstr] if isinstance(reconstr, str) else reconstr
    m.limiter = LIM[limiter] if isinstance(limiter, str) else limiter
    m.charact_proj = charact_proj
    m.kappa0, m.thcond_type, m.sat_hfe, m.cour_diff = kappa0, TC[thcond_type], sat_hfe, cour_diff
    m.fixdt, m.dt_fixed = int(bool(fixdt)), dt_fixed
    m.outflow_face_aware, m.exact_fp = outflow_face_aware, int(bool(exact_fp))
    m.path = PATH[path] if isinstance(path, str) else path
    for a in range(3):
        m.grav[a] = grav[a]
    m.drive_f0, m.drive_tau, m.drive_nmod, m.drive_seed = drive_f0, drive_tau, drive_nmod, drive_seed
    m.hydro = int(bool(hydro))
    return m


_GRID_KEYS = ("Nx", "Ny", "Nz", "dims", "lmin", "lmax", "bc")


class Context:
    """One grid on the device (owns a bnz_ctx, or views an instance of a Batch).

    path: "fused" (the tile kernels: fastest for 2D PLM grids), "split" (per-axis
    flux kernels and one fused update per stage: fastest for 1D and 3D grids) or
    "plain" (one kernel per loop of the reference).  The hydro build runs on
    "plain" and "split".
    The three give the same bits with exact_fp=True."""

    def __init__(self, Nx=None, Ny=1, Nz=1, dims=2, lmin=(0., 0., 0.), lmax=(1., 1., 1.),
                 bc=((0, 0), (0, 0), (0, 0)), _handle=None, _owner=None, **method):
        self.L = load()
        if _handle is not None:
            self.h, self._owner, self._owns = _handle, _owner, False
        else:
            g = grid_desc(Nx, Ny, Nz, dims, lmin, lmax, bc)
            m = method_desc(**method)
            self.grid_desc, self.method_desc = g, m
            h = C.c_void_p()
            rc = self.L.bnz_create(C.byref(g), C.byref(m), C.byref(h))
            self.h, self._owner, self._owns = h, None, True
            if rc != BNZ_OK:
                msg = self.L.bnz_last_error(h).decode() if h.value else "bnz_create failed"
                self.L.bnz_destroy(h)
                self.h = C.c_void_p()
                raise BnzError(rc, msg)
        nt = (C.c_int * 3)()
        ng = C.c_int()
        self.L.bnz_shape(self.h, nt, C.byref(ng))
        self.shape = (nt[2], nt[1], nt[0])
        self.ng = ng.value

    def _ck(self, rc):
        if rc != BNZ_OK:
            raise BnzError(rc, self.L.bnz_last_error(self.h).decode())

    def close(self):
        if getattr(self, "_owns", False) and self.h.value:
            self.L.bnz_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, prim_or_cons, bfld=None, is_prim=True):
        a = np.ascontiguousarray(prim_or_cons, dtype=np.float64)
        if a.shape != (9,) + self.shape:
            raise ValueError("state must have shape %s" % ((9,) + self.shape,))
        b = None
        if bfld is not None:
            b = np.ascontiguousarray(bfld, dtype=np.float64)
            if b.shape != (3,) + self.shape:
                raise ValueError("bfld must have shape %s" % ((3,) + self.shape,))
        self._ck(self.L.bnz_set_state(self.h, _p(a), int(bool(is_prim)), _p(b)))

    def init(self):
        self._ck(self.L.bnz_init(self.h))

    def get_state(self, prim=True, cons=True, bfld=True):
        P = np.empty((9,) + self.shape) if prim else None
        U = np.empty((9,) + self.shape) if cons else None
        B = np.empty((3,) + self.shape) if bfld else None
        self._ck(self.L.bnz_get_state(self.h, _p(P), _p(U), _p(B)))
        return P, U, B

    def get_state_into(self, prim=None, cons=None, bfld=None):
        """Download into caller-provided float64 arrays (e.g. pinned buffers)."""
        for a, nv in ((prim, 9), (cons, 9), (bfld, 3)):
            if a is not None and (a.shape != (nv,) + self.shape or a.dtype != np.float64
                                  or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("output array has the wrong shape or layout")
        self._ck(self.L.bnz_get_state(self.h, _p(prim), _p(cons), _p(bfld)))

    def apply_bc(self, mask=0xFFF):
        self._ck(self.L.bnz_apply_bc(self.h, mask))

    def new_dt(self):
        dt = C.c_double()
        self._ck(self.L.bnz_new_dt(self.h, C.byref(dt)))
        return dt.value

    def step(self, dt):
        self._ck(self.L.bnz_vl2_step(self.h, dt))

    def diffuse(self, dt):
        n = C.c_int()
        self._ck(self.L.bnz_diffuse(self.h, dt, C.byref(n)))
        return n.value

    def advance(self, tmax, max_steps=0):
        t = C.c_double()
        s = C.c_long()
        self._ck(self.L.bnz_advance(self.h, tmax, max_steps, C.byref(t), C.byref(s)))
        return t.value, s.value

    def last_nsts(self):
        n = C.c_int()
        self._ck(self.L.bnz_last_nsts(self.h, C.byref(n)))
        return n.value

    def set_time(self, time, step):
        self._ck(self.L.bnz_set_time(self.h, float(time), int(step)))

    def time(self):
        t, s, d = C.c_double(), C.c_long(), C.c_double()
        self._ck(self.L.bnz_get_time(self.h, C.byref(t), C.byref(s), C.byref(d)))
        return t.value, s.value, d.value

    def check(self):
        """Raises BnzError(BNZ_ERR_STATE) if the device flagged a non-physical state."""
        bits = C.c_uint32()
        self._ck(self.L.bnz_check(self.h, C.byref(bits)))
        return bits.value

    def sync(self):
        self._ck(self.L.bnz_sync(self.h))

    def advance_graph(self, tmax, nsteps):
        self._ck(self.L.bnz_advance_graph(self.h, tmax, nsteps))

    def device_state(self):
        p, u, b = _dp(), _dp(), _dp()
        self._ck(self.L.bnz_device_state(self.h, C.byref(p), C.byref(u), C.byref(b)))
        return (C.cast(p, C.c_void_p).value, C.cast(u, C.c_void_p).value, C.cast(b, C.c_void_p).value)

    # --- output support ---------------------------------------------------
    def history(self):
        """The reference's 16-column history row (output.pyx get_hst_vars_grid)."""
        out = np.zeros(16)
        self._ck(self.L.bnz_history(self.h, _p(out)))
        return out

    def div_b(self):
        """max |div B| * dx / max |B| over the active cells, reduced on the device."""
        out = np.zeros(2)
        self._ck(self.L.bnz_div_b(self.h, _p(out)))
        return out[0] / out[1] if out[1] > 0 else out[0]

    def snapshot(self, prim=None, cons=None, bfld=None):
        """Queue a device->host copy of the state into the given float64 arrays
        (keep them alive, ideally page-locked, until snapshot_wait())."""
        for a, nv in ((prim, 9), (cons, 9), (bfld, 3)):
            if a is not None and (a.shape != (nv,) + self.shape or a.dtype != np.float64
                                  or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("snapshot array has the wrong shape or layout")
        self._ck(self.L.bnz_snapshot(self.h, _p(prim), _p(cons), _p(bfld)))

    def snapshot_wait(self):
        self._ck(self.L.bnz_snapshot_wait(self.h))

    # --- device-pointer state and the adjoint (pointers are ints) ---------
    def set_state_device(self, prim_ptr, bfld_ptr):
        self._ck(self.L.bnz_set_state_device(self.h, C.c_void_p(prim_ptr), C.c_void_p(bfld_ptr)))

    def get_state_device(self, prim_ptr, bfld_ptr):
        self._ck(self.L.bnz_get_state_device(self.h, C.c_void_p(prim_ptr), C.c_void_p(bfld_ptr)))

    def rollout_forward(self, nsteps, dt, checkpoint_every=10):
        self._ck(self.L.bnz_rollout_forward(self.h, int(nsteps), float(dt), int(checkpoint_every)))

    def rollout_adjoint(self, gprim_ptr, gbfld_ptr, gprim0_ptr, gbfld0_ptr):
        self._ck(self.L.bnz_rollout_adjoint(self.h, C.c_void_p(gprim_ptr), C.c_void_p(gbfld_ptr),
                                            C.c_void_p(gprim0_ptr), C.c_void_p(gbfld0_ptr)))

    def step_adjoint(self, dt, prim_ptr, bfld_ptr, gprim1_ptr, gbfld1_ptr, gprim0_ptr, gbfld0_ptr):
        self._ck(self.L.bnz_step_adjoint(self.h, float(dt), C.c_void_p(prim_ptr), C.c_void_p(bfld_ptr),
                                         C.c_void_p(gprim1_ptr), C.c_void_p(gbfld1_ptr),
                                         C.c_void_p(gprim0_ptr), C.c_void_p(gbfld0_ptr)))

    def set_stream(self, stream):
        """Order this context's work on a caller-owned CUDA stream (handle as int)."""
        self._ck(self.L.bnz_set_stream(self.h, C.c_void_p(stream)))

    def launch_count(self):
        n = C.c_longlong()
        self._ck(self.L.bnz_launch_count(self.h, C.byref(n)))
        return n.value

    def stream(self):
        s = C.c_void_p()
        self._ck(self.L.bnz_stream(self.h, C.byref(s)))
        return s.value


class Batch:
    """Many independent grids of uneven size with one method (bnz_batch_* in
    include/bnz_gpu.h): 2D grids by one launch per stage over every instance,
    3D grids likewise on the fused chunk kernels, or with path="split" on the
    split path one instance after another."""

    def __init__(self, grids, **method):
        self.L = load()
        n = len(grids)
        arr = (GridDesc * n)()
        for q, gkw in enumerate(grids):
            arr[q] = grid_desc(**gkw)
        m = method_desc(**method)
        h = C.c_void_p()
        rc = self.L.bnz_batch_create(arr, n, C.byref(m), C.byref(h))
        self.h = h
        if rc != BNZ_OK:
            msg = self.L.bnz_batch_last_error(h).decode() if h.value else "bnz_batch_create failed"
            self.L.bnz_batch_destroy(h)
            self.h = C.c_void_p()
            raise BnzError(rc, msg)
        self.instances = []
        for q in range(n):
            ch = C.c_void_p()
            self._ck(self.L.bnz_batch_instance(h, q, C.byref(ch)))
            self.instances.append(Context(_handle=ch, _owner=self))

    def _ck(self, rc):
        if rc != BNZ_OK:
            raise BnzError(rc, self.L.bnz_batch_last_error(self.h).decode())

    def __len__(self):
        return len(self.instances)

    def __getitem__(self, i):
        return self.instances[i]

    def advance(self, tmax, nsteps):
        self._ck(self.L.bnz_batch_advance(self.h, tmax, nsteps))

    def advance_timed(self, tmax, nsteps):
        """advance() launched one by one with events around every launch:
        returns the mean ms per launch of the dt, predictor and corrector kernels."""
        ms = (C.c_double * 3)()
        self._ck(self.L.bnz_batch_advance_timed(self.h, tmax, int(nsteps), ms))
        return {"dt": ms[0], "predictor": ms[1], "corrector": ms[2]}

    def step_host(self, prims, bflds, tmax=1e30, nsteps=1, nchunks=0):
        """Load every instance's state from the host arrays, advance nsteps
        steps and write the result (ghosts filled) back into the same arrays.
        Copies in, steps and copies out of groups of instances overlap
        (bnz_batch_step_host); pinned arrays make the copies asynchronous."""
        n = len(self.instances)
        if len(prims) != n or len(bflds) != n:
            raise ValueError("one prim and one bfld array per instance")
        arrays = list(prims) + list(bflds)
        cached = getattr(self, "_host_ptrs", None)
        if cached is None or any(x is not y for x, y in zip(cached[0], arrays)):
            pp, pb = (_dp * n)(), (_dp * n)()
            for q, (c, P, B) in enumerate(zip(self.instances, prims, bflds)):
                for a, nv in ((P, 9), (B, 3)):
                    if (a.shape != (nv,) + c.shape or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]
                            or not a.flags["WRITEABLE"]):
                        raise ValueError("state array of instance %d has the wrong shape or layout" % q)
                pp[q] = P.ctypes.data_as(_dp)
                pb[q] = B.ctypes.data_as(_dp)
            # the same array objects (held here) reuse the pointer tables of the last call
            cached = self._host_ptrs = (arrays, pp, pb)
        self._ck(self.L.bnz_batch_step_host(self.h, cached[1], cached[2], float(tmax), int(nsteps), int(nchunks)))

    def set_stream(self, stream):
        self._ck(self.L.bnz_batch_set_stream(self.h, C.c_void_p(stream)))

    def test_withhold_loads(self, on):
        """Test switch: the persistent kernels' TMA loads are armed but not
        issued, so their bounded waits run out (bnz_batch_test_withhold_loads)."""
        self._ck(self.L.bnz_batch_test_withhold_loads(self.h, int(bool(on))))

    def launch_count(self):
        n = C.c_longlong()
        self._ck(self.L.bnz_batch_launch_count(self.h, C.byref(n)))
        return n.value

    def sync(self):
        self._ck(self.L.bnz_batch_sync(self.h))

    @property
    def variant(self):
        v = C.c_int()
        self._ck(self.L.bnz_batch_get_variant(self.h, C.byref(v)))
        return v.value

    def set_variant(self, v):
        self._ck(self.L.bnz_batch_set_variant(self.h, int(v)))

    def time_variant(self, v, steps=2):
        """ms per batch step of variant v (state restored afterwards)."""
        ms = C.c_double()
        self._ck(self.L.bnz_batch_time_variant(self.h, int(v), int(steps), C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            for c in self.instances:
                c.h = C.c_void_p()
            self.L.bnz_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def riemann(rsolver, wl, wr, bx, gam, exact_fp=False):
    """Device Riemann fluxes of face states given as torch CUDA float64 tensors
    of shape (nvar, n) (bnz_riemann: the reference's C-level flux call, nvar 9
    for MHD, 6 for the hydro build).  Returns the flux tensor."""
    import torch
    L = load()
    nvar, n = wl.shape
    wl, wr = wl.contiguous(), wr.contiguous()
    bx = bx.contiguous() if bx is not None else None
    flux = torch.empty_like(wl)
    err = torch.zeros(1, dtype=torch.int32, device=wl.device)
    rs = RS[rsolver] if isinstance(rsolver, str) else rsolver
    rc = L.bnz_riemann(rs, nvar, wl.data_ptr(), wr.data_ptr(), bx.data_ptr() if bx is not None else None,
                       flux.data_ptr(), n, float(gam), int(bool(exact_fp)), err.data_ptr(),
                       torch.cuda.current_stream().cuda_stream)
    if rc != BNZ_OK:
        raise BnzError(rc, "bnz_riemann failed")
    return flux


def fp64_fma_peak():
    """Measured FP64 FMA throughput of the current device, TFLOP/s."""
    L = load()
    t = C.c_double()
    rc = L.bnz_fp64_fma_peak(C.byref(t))
    if rc != BNZ_OK:
        raise BnzError(rc, "bnz_fp64_fma_peak failed")
    return t.value


def fast_rcp(x):
    """1 / x (a CUDA float64 tensor) by the fast build's Newton-refined reciprocal."""
    import torch
    L = load()
    x = x.contiguous()
    y = torch.empty_like(x)
    rc = L.bnz_fast_rcp(x.data_ptr(), y.data_ptr(), x.numel(), torch.cuda.current_stream().cuda_stream)
    if rc != BNZ_OK:
        raise BnzError(rc, "bnz_fast_rcp failed")
    return y


def variants():
    """[(tx, ty, staged, persistent)] of the fused kernel variants."""
    L = load()
    n = C.c_int()
    L.bnz_variant_count(C.byref(n), None, None, None, None)
    tx, ty, st, pe = [(C.c_int * n.value)() for _ in range(4)]
    L.bnz_variant_count(C.byref(n), tx, ty, st, pe)
    return [(tx[v], ty[v], st[v], pe[v]) for v in range(n.value)]


def variant_label(v):
    """'15x14s' style name of a variant tuple: s = staged predictor, p = persistent
    corrector, pp = persistent predictor and corrector."""
    return "%dx%d%s%s" % (v[0], v[1], "s" if v[2] else "", "p" * v[3])
