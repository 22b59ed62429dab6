"""torch.autograd wrapper around the hand-written adjoint -- for gradient checks only.

`rollout(...)` runs `nsteps` explicit substeps through the C ABI
(mpm_diff_forward) and returns the final particle state; its backward calls
mpm_diff_backward (hand-written CUDA adjoint kernels, checkpointed every
`checkpoint_every` substeps).  Arrays stay on the GPU; torch only carries the
gradients between the loss and the kernels.
"""
from __future__ import annotations

import torch

from . import driver as D


def _colmajor(M):          # (n,3,3) row-major -> (n,9) column-major per particle
    return M.transpose(1, 2).reshape(M.shape[0], -1).contiguous()


def _rowmajor(Mc):         # inverse of _colmajor
    n = Mc.shape[0]
    return Mc.reshape(n, 3, 3).transpose(1, 2).contiguous()


class MPMRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, X, V, F, B, mu, lam, drv, mass, volume, nsteps, checkpoint_every):
        drv.set_particles_device(X.detach().contiguous(), V.detach().contiguous(), _colmajor(F.detach()),
                                 _colmajor(B.detach()), mass, volume, mu.detach().contiguous(),
                                 lam.detach().contiguous())
        drv.diff_forward(nsteps, checkpoint_every)
        X1, V1, F1c, B1c, valid = drv.get_particles_device(X.dtype)
        ctx.drv = drv
        ctx.mark_non_differentiable(valid)
        return X1, V1, _rowmajor(F1c), _rowmajor(B1c), valid

    @staticmethod
    def backward(ctx, gX, gV, gF, gB, gvalid):
        drv = ctx.drv
        z = lambda g, shape: torch.zeros(shape, dtype=drv_dtype(drv), device="cuda") if g is None else g
        n = drv.n
        gX = z(gX, (n, 3)).contiguous()
        gV = z(gV, (n, 3)).contiguous()
        gF = _colmajor(z(gF, (n, 3, 3)))
        gB = _colmajor(z(gB, (n, 3, 3)))
        aX, aV, aFc, aBc, amu, alam = drv.diff_backward(gX, gV, gF, gB)
        return aX, aV, _rowmajor(aFc), _rowmajor(aBc), amu, alam, None, None, None, None, None


def drv_dtype(drv):
    return torch.float64 if drv.precision == D.FP64 else torch.float32


def rollout(drv, X, V, F, B, mu, lam, mass, volume, nsteps, checkpoint_every=8):
    return MPMRollout.apply(X, V, F, B, mu, lam, drv, mass, volume, nsteps, checkpoint_every)


def com_loss(X, mass, target):
    """Squared distance of the final mass-weighted centre of mass to `target`.

    Internal forces conserve momentum, so without collision objects this loss
    depends on v0 and gravity only; its gradient w.r.t. E is zero."""
    com = (mass[:, None] * X).sum(0) / mass.sum()
    return ((com - target) ** 2).sum()


def part_com_loss(X, mass, part, target):
    """Same loss for the centre of mass of a subset `part` (bool mask) of the
    particles; it moves with the body's deformation, so it depends on E."""
    m = mass * part
    com = (m[:, None] * X).sum(0) / m.sum()
    return ((com - target) ** 2).sum()
