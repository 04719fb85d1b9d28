"""The VL2 step that allocates no device memory (bnz_vl2_step_noalloc).

Some callers cannot let a library call cudaMalloc: their device memory is
handed out by a framework allocator that reserved it up front, or their time
loop must not meet the device-wide synchronisation an allocation implies.
They own the input and output buffers; the step keeps its own working memory
in a fixed device array inside the library.  This file runs last (pytest
collects files in name order) and checks the entry point, through the C ABI,
against the regular context step, two calls in a row -- run alone in a fresh
process or after the other tests.
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
    return lib, L


@pytest.mark.parametrize("case,n,kw", [("blast", 48, {}), ("vortex", 64, dict(limiter="mc")),
                                       ("blast_reflect", 40, dict(rsolver="hll"))])
def test_noalloc_step_matches_context_step(case, n, kw):
    import torch
    lib, L = _abi()
    gc, prim, bfld, opts = setup_case(case, n=n)
    ref = device_ctx(opts, path="fused", **kw)
    ref.set_state(prim, bfld)
    ref.init()
    P0, _, B0 = ref.get_state()
    dt = ref.new_dt()
    # the caller owns the device buffers; the entry point allocates nothing
    a_p = torch.from_numpy(P0).cuda()
    a_b = torch.from_numpy(B0).cuda()
    b_p = torch.zeros_like(a_p)
    b_b = torch.zeros_like(a_b)
    g = lib.grid_desc(**{k: opts[k] for k in ("Nx", "Ny", "Nz", "dims", "bc")})
    m = lib.method_desc(**{k: v for k, v in dict(opts, **kw).items()
                           if k not in ("Nx", "Ny", "Nz", "dims", "bc")})
    stream = torch.cuda.current_stream().cuda_stream
    for src_p, src_b, dst_p, dst_b in ((a_p, a_b, b_p, b_b), (b_p, b_b, a_p, a_b)):
        rc = L.bnz_vl2_step_noalloc(C.byref(g), C.byref(m), src_p.data_ptr(), src_b.data_ptr(),
                                    dst_p.data_ptr(), dst_b.data_ptr(), dt, stream)
        assert rc == 0, L.bnz_noalloc_last_error().decode()
        ref.step(dt)
    torch.cuda.synchronize()
    P1, _, B1 = ref.get_state()
    # same kernels as the context's fused step: the results agree bit for bit
    assert np.array_equal(a_p.cpu().numpy(), P1)
    assert np.array_equal(a_b.cpu().numpy(), B1)
    assert ref.check() == 0


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    lib, L = _abi()
    assert L.bnz_noalloc_scratch_bytes() == 4 << 20
    g = lib.grid_desc(Nx=400, Ny=400, Nz=1, dims=2, bc=((1, 1), (1, 1), (0, 0)))
    m = lib.method_desc()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = L.bnz_vl2_step_noalloc(C.byref(g), C.byref(m), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                x.data_ptr(), 1e-3, None)
    assert rc == lib.BNZ_ERR_ARG
    assert "too large" in L.bnz_noalloc_last_error().decode()
