"""The C-ABI library loads, exports every symbol include/bnz_gpu.h declares and
rejects bad configurations on the host before any device call (CPU-only)."""
import ctypes as C
import os
import re

import pytest

from bonzo_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:int|const char\*|void|size_t)\s+(bnz_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_header_and_binding_agree():
    assert sorted(_lib.EXPORTS) == [n for n in header_functions() if n in _lib.EXPORTS]
    assert set(header_functions()) >= set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIB_PATH)
    for name in header_functions():
        assert hasattr(L, name), name


def _try_create(**kw):
    g = _lib.GridDesc()
    m = _lib.MethodDesc()
    base = dict(Nx=16, Ny=16, Nz=1, dims=2)
    base.update({k: v for k, v in kw.items() if k in ("Nx", "Ny", "Nz", "dims")})
    g.Nx, g.Ny, g.Nz, g.dims = base["Nx"], base["Ny"], base["Nz"], base["dims"]
    for a in range(3):
        g.lmax[a] = 1.0
    for a, sides in enumerate(kw.get("bc", ((0, 0), (0, 0), (0, 0)))):
        g.bc[a][0], g.bc[a][1] = sides
    m.gam, m.cour = kw.get("gam", 5. / 3), kw.get("cour", 0.4)
    m.rsolver, m.reconstr, m.limiter = kw.get("rsolver", 2), 1, kw.get("limiter", 0)
    m.charact_proj = kw.get("charact_proj", 0)
    m.kappa0, m.cour_diff = kw.get("kappa0", 0.), 0.5
    m.path = kw.get("path", 1)
    m.hydro = kw.get("hydro", 0)
    L = _lib.load()
    h = C.c_void_p()
    rc = L.bnz_create(C.byref(g), C.byref(m), C.byref(h))
    msg = L.bnz_last_error(h).decode() if h.value else ""
    if h.value:
        L.bnz_destroy(h)
    return rc, msg


@pytest.mark.parametrize("kw,frag", [
    (dict(dims=4), "dims"),
    (dict(dims=2, Nz=4), "Nz>1"),
    (dict(gam=1.0), "gam"),
    (dict(cour=0.0), "cour"),
    (dict(rsolver=1), "hllc"),
    (dict(limiter=7), "limiter"),
    (dict(bc=((0, 1), (0, 0), (0, 0))), "periodic"),
    (dict(kappa0=-1.0), "kappa0"),
    (dict(Nx=2), "ng"),
    (dict(path=5), "path"),
    (dict(hydro=1, rsolver=2), "hydro mode"),
    (dict(hydro=1, rsolver=1, path=0), "plain path"),
    (dict(hydro=1, rsolver=1, charact_proj=1), "charact_proj"),
    (dict(hydro=1, rsolver=0, kappa0=0.1), "conduction"),
    (dict(hydro=3, rsolver=1), "hydro"),
])
def test_bad_config_rejected_on_host(kw, frag):
    rc, msg = _try_create(**kw)
    assert rc == _lib.BNZ_ERR_ARG
    assert frag in msg


def test_riemann_entry_rejects_bad_arguments_on_host():
    """bnz_riemann checks its arguments before any device call: hllc is the
    hydro build's (nvar 6), hlld the MHD builds' (nvar 9)."""
    L = _lib.load()
    p = C.c_void_p(16)  # never dereferenced: every case fails its host checks
    assert L.bnz_riemann(1, 9, p, p, p, p, 4, 5. / 3, 0, None, None) == _lib.BNZ_ERR_UNSUPPORTED
    assert L.bnz_riemann(2, 6, p, p, p, p, 4, 5. / 3, 0, None, None) == _lib.BNZ_ERR_UNSUPPORTED
    assert L.bnz_riemann(0, 7, p, p, p, p, 4, 5. / 3, 0, None, None) == _lib.BNZ_ERR_ARG
    assert L.bnz_riemann(0, 9, p, p, None, p, 4, 5. / 3, 0, None, None) == _lib.BNZ_ERR_ARG
    assert L.bnz_riemann(0, 9, p, p, p, p, -1, 5. / 3, 0, None, None) == _lib.BNZ_ERR_ARG
    assert L.bnz_riemann(0, 9, p, p, p, p, 0, 5. / 3, 0, None, None) == _lib.BNZ_OK


def test_null_arguments():
    L = _lib.load()
    assert L.bnz_create(None, None, None) == _lib.BNZ_ERR_ARG
    assert L.bnz_vl2_step(None, 0.1) == _lib.BNZ_ERR_ARG
    assert L.bnz_destroy(None) == _lib.BNZ_OK


def test_kernel_variants_and_their_labels():
    """The autotuner's candidates (host-only query): tile shapes, predictor
    staging, persistent kernels; every variant has its own label, so timings
    keyed by label cannot overwrite each other."""
    vs = _lib.variants()
    assert len(vs) == 10
    assert vs[0] == (32, 8, 0, 0)            # a single grid's default
    assert vs[8] == (15, 14, 0, 2)           # a batch's default: persistent predictor and corrector
    assert vs[9] == (14, 14, 0, 2)
    assert [v[3] for v in vs].count(0) == 6 and [v[3] for v in vs].count(1) == 2
    labels = [_lib.variant_label(v) for v in vs]
    assert len(set(labels)) == len(labels)
    assert labels[8] == "15x14pp" and labels[6] == "15x14p" and labels[1] == "32x8s"
