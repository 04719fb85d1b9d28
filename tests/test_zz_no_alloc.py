"""The VL2 step that allocates no device memory (bnz_vl2_step_noalloc).

Some callers cannot let a library call cudaMalloc: their device memory is
handed out by a framework allocator that reserved it up front, or their time
loop must not meet the device-wide synchronisation an allocation implies.
They own the input and output buffers; the step keeps its own working memory
in a fixed device array inside the library.  This file runs last (pytest
collects files in name order) and checks the entry point, through the C ABI,
against the regular context step, two calls in a row -- run alone in a fresh
process or after the other tests.  It also checks the sticky error word that
bnz_noalloc_check reads back, with a non-physical state planted on the host.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import device_ctx, setup_case

pytestmark = pytest.mark.gpu


def _abi():
    from bonzo_b200 import _lib as lib
    L = lib.load()
    L.bnz_vl2_step_noalloc.argtypes = [C.POINTER(lib.GridDesc), C.POINTER(lib.MethodDesc), C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
    L.bnz_noalloc_last_error.restype = C.c_char_p
    L.bnz_noalloc_scratch_bytes.restype = C.c_size_t
    L.bnz_noalloc_check.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    return lib, L


class _Case:
    """A grid, its context (the regular step) and the caller-owned buffers."""

    def __init__(self, lib, case, n, kw):
        import torch
        gc, prim, bfld, opts = setup_case(case, n=n)
        self.ref = device_ctx(opts, path="fused", **kw)
        self.ref.set_state(prim, bfld)
        self.ref.init()
        P0, _, B0 = self.ref.get_state()
        self.dt = self.ref.new_dt()
        self.a_p = torch.from_numpy(P0).cuda()
        self.a_b = torch.from_numpy(B0).cuda()
        self.b_p = torch.zeros_like(self.a_p)
        self.b_b = torch.zeros_like(self.a_b)
        self.g = lib.grid_desc(**{k: opts[k] for k in ("Nx", "Ny", "Nz", "dims", "bc")})
        self.m = lib.method_desc(**{k: v for k, v in dict(opts, **kw).items()
                                    if k not in ("Nx", "Ny", "Nz", "dims", "bc")})
        self.k = 0

    def step(self, L, stream):
        """One no-alloc step from the current buffer pair into the other, and
        one context step."""
        src = (self.a_p, self.a_b) if self.k % 2 == 0 else (self.b_p, self.b_b)
        dst = (self.b_p, self.b_b) if self.k % 2 == 0 else (self.a_p, self.a_b)
        rc = L.bnz_vl2_step_noalloc(C.byref(self.g), C.byref(self.m), src[0].data_ptr(), src[1].data_ptr(),
                                    dst[0].data_ptr(), dst[1].data_ptr(), self.dt, stream)
        assert rc == 0, L.bnz_noalloc_last_error().decode()
        self.ref.step(self.dt)
        self.k += 1
        return dst

    def same_as_context(self, dst):
        P1, _, B1 = self.ref.get_state()
        return np.array_equal(dst[0].cpu().numpy(), P1) and np.array_equal(dst[1].cpu().numpy(), B1)


def _check(L, stream):
    bits = C.c_uint32()
    rc = L.bnz_noalloc_check(stream, C.byref(bits))
    return rc, bits.value


CASES = [("blast", 48, {}), ("vortex", 64, dict(limiter="mc")), ("blast_reflect", 40, dict(rsolver="hll")),
         ("vortex", 40, dict(rsolver="hllt")), ("blast_reflect", 32, dict(grav=(0.0, -1.0, 0.0))),
         ("vortex_pert", 40, dict(limiter="mc", charact_proj=1)), ("blast", 36, dict(exact_fp=True))]


@pytest.mark.parametrize("case,n,kw", CASES)
def test_noalloc_step_matches_context_step(case, n, kw):
    import torch
    lib, L = _abi()
    stream = torch.cuda.current_stream().cuda_stream
    _check(L, stream)  # start from a clear error word
    c = _Case(lib, case, n, kw)
    for _ in range(2):
        dst = c.step(L, stream)
    torch.cuda.synchronize()
    # same kernels as the context's fused step: the results agree bit for bit
    assert c.same_as_context(dst)
    assert c.ref.check() == 0
    assert _check(L, stream) == (0, 0)


def test_noalloc_alternating_grid_sizes():
    """Back-to-back calls on two grids of different sizes: each call rebuilds
    its descriptor, tiles and coordinates in the shared array."""
    import torch
    lib, L = _abi()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [_Case(lib, "blast", 48, {}), _Case(lib, "vortex", 70, {})]
    for _ in range(2):
        for c in cases:
            dst = c.step(L, stream)
            torch.cuda.synchronize()
            assert c.same_as_context(dst)
    assert _check(L, stream) == (0, 0)


def test_noalloc_reports_a_nonphysical_state():
    """A negative pressure planted in the input: the step's error word is
    raised, bnz_noalloc_check reports it (with the context path's bits) and
    clears it."""
    import torch
    lib, L = _abi()
    stream = torch.cuda.current_stream().cuda_stream
    _check(L, stream)
    gc, prim, bfld, opts = setup_case("blast", n=40)
    prim[4][0, gc.j1 + 20, gc.i1 + 3] = -1.0
    c = _Case.__new__(_Case)
    c.ref = device_ctx(opts, path="fused")
    c.ref.set_state(prim, bfld)
    c.ref.init()
    P0, _, B0 = c.ref.get_state()
    c.dt = 1e-4
    c.a_p, c.a_b = torch.from_numpy(P0).cuda(), torch.from_numpy(B0).cuda()
    c.b_p, c.b_b = torch.zeros_like(c.a_p), torch.zeros_like(c.a_b)
    c.g = lib.grid_desc(**{k: opts[k] for k in ("Nx", "Ny", "Nz", "dims", "bc")})
    c.m = lib.method_desc(**{k: v for k, v in opts.items() if k not in ("Nx", "Ny", "Nz", "dims", "bc")})
    c.k = 0
    c.step(L, stream)
    rc, bits = _check(L, stream)
    assert rc == lib.BNZ_ERR_STATE and bits != 0
    ref_bits = C.c_uint32()
    L.bnz_check(c.ref.h, C.byref(ref_bits))
    assert bits == ref_bits.value
    assert _check(L, stream) == (0, 0)


def test_noalloc_rejects_bad_arguments():
    import torch
    lib, L = _abi()
    assert L.bnz_noalloc_scratch_bytes() == 4 << 20
    m = lib.method_desc()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    g = lib.grid_desc(Nx=400, Ny=400, Nz=1, dims=2, bc=((1, 1), (1, 1), (0, 0)))
    rc = L.bnz_vl2_step_noalloc(C.byref(g), C.byref(m), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                x.data_ptr(), 1e-3, None)
    assert rc == lib.BNZ_ERR_ARG
    assert "too large" in L.bnz_noalloc_last_error().decode()
    # in place (output == input) is refused before any launch
    g = lib.grid_desc(Nx=16, Ny=16, Nz=1, dims=2, bc=((1, 1), (1, 1), (0, 0)))
    n = 22 * 22
    p = torch.zeros(9 * n, dtype=torch.float64, device="cuda")
    b = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    q = torch.zeros(9 * n, dtype=torch.float64, device="cuda")
    rc = L.bnz_vl2_step_noalloc(C.byref(g), C.byref(m), p.data_ptr(), b.data_ptr(), p.data_ptr(),
                                b.data_ptr(), 1e-3, None)
    assert rc == lib.BNZ_ERR_ARG and "overlap" in L.bnz_noalloc_last_error().decode()
    rc = L.bnz_vl2_step_noalloc(C.byref(g), C.byref(m), p.data_ptr(), b.data_ptr(), q.data_ptr(),
                                q.data_ptr() + 8 * 9 * n - 64, 1e-3, None)
    assert rc == lib.BNZ_ERR_ARG and "overlap" in L.bnz_noalloc_last_error().decode()
    # a 2D grid needs a positive z depth
    g = lib.grid_desc(Nx=16, Ny=16, Nz=1, dims=2, lmax=(1., 1., 0.), bc=((1, 1), (1, 1), (0, 0)))
    rc = L.bnz_vl2_step_noalloc(C.byref(g), C.byref(m), p.data_ptr(), b.data_ptr(), q.data_ptr(),
                                q.data_ptr(), 1e-3, None)
    assert rc == lib.BNZ_ERR_ARG and "lmax" in L.bnz_noalloc_last_error().decode()
