"""Differentiable VL2 rollouts: torch.autograd.Function over the hand-written
discrete adjoint (bnz_rollout_forward / bnz_rollout_adjoint in
include/bnz_gpu.h).

    eng = bonzo_b200.Context(Nx=256, Ny=256, dims=2, bc=..., path="fused", ...)
    prim_T, bfld_T = rollout(prim0, bfld0, eng, nsteps=100, dt=1e-4, checkpoint_every=10)
    loss = ((prim_T[0] - rho_target) ** 2).sum()
    loss.backward()            # prim0.grad, bfld0.grad

prim0 (9, Ntot...) and bfld0 (3, Ntot...) are float64 CUDA tensors with the
context's full shape (ghosts included).  The forward reads only the source
entries of the input (active cells and the faces the CT update owns); the
gradient is zero on the ghost entries.  dt is held fixed: the gradient does not
differentiate a CFL time step.  Work is ordered on torch's current stream.

The context must use the fused 2D path with rsolver hll, hllt or hlld; any
limiter (with or without charact_proj), any boundary conditions and constant
gravity are differentiated.  Conduction (kappa0 > 0) and turbulence driving
are refused with BnzError (unsupported).
"""
import torch

from ._lib import Context


def _check(t, nv, eng):
    if not (t.is_cuda and t.dtype == torch.float64):
        raise TypeError("state tensors must be float64 CUDA tensors")
    if tuple(t.shape) != (nv,) + tuple(eng.shape):
        raise ValueError("expected shape %s, got %s" % ((nv,) + tuple(eng.shape), tuple(t.shape)))
    return t.contiguous()


class VL2Rollout(torch.autograd.Function):
    """nsteps VL2 steps of fixed dt; backward runs the adjoint with
    checkpoint-and-recompute every `checkpoint_every` steps."""

    @staticmethod
    def forward(ctx, prim0, bfld0, eng, nsteps, dt, checkpoint_every):
        prim0 = _check(prim0, 9, eng)
        bfld0 = _check(bfld0, 3, eng)
        eng.set_stream(torch.cuda.current_stream().cuda_stream)
        eng.set_state_device(prim0.data_ptr(), bfld0.data_ptr())
        eng.rollout_forward(nsteps, dt, checkpoint_every)
        prim = torch.empty_like(prim0)
        bfld = torch.empty_like(bfld0)
        eng.get_state_device(prim.data_ptr(), bfld.data_ptr())
        ctx.eng = eng
        return prim, bfld

    @staticmethod
    def backward(ctx, gprim, gbfld):
        eng = ctx.eng
        gprim = torch.zeros(eng_shape(eng, 9), dtype=torch.float64, device="cuda") if gprim is None \
            else gprim.contiguous().clone()
        gbfld = torch.zeros(eng_shape(eng, 3), dtype=torch.float64, device="cuda") if gbfld is None \
            else gbfld.contiguous().clone()
        g0 = torch.empty_like(gprim)
        b0 = torch.empty_like(gbfld)
        eng.set_stream(torch.cuda.current_stream().cuda_stream)
        eng.rollout_adjoint(gprim.data_ptr(), gbfld.data_ptr(), g0.data_ptr(), b0.data_ptr())
        return g0, b0, None, None, None, None


def eng_shape(eng, nv):
    return (nv,) + tuple(eng.shape)


def rollout(prim0, bfld0, eng, nsteps, dt, checkpoint_every=10):
    """Differentiable rollout through the context `eng` (a fused-path Context)."""
    if not isinstance(eng, Context):
        raise TypeError("eng must be a bonzo_b200 Context")
    return VL2Rollout.apply(prim0, bfld0, eng, int(nsteps), float(dt), int(checkpoint_every))
