"""torch.autograd bridge: the waveform misfit as a differentiable function of Vp, Vs, rho
and the moment tensors, with the exact adjoint of libefm as its backward.

    J = ElasticMisfit.apply(vp, vs, rho, mt, batch, obs)
    J.backward()          # vp.grad, vs.grad, rho.grad, mt.grad

J = 0.5 * sum over every instance of (modelled - observed)^2 (float64), the misfit of
computeCostFunction (mainPropElastic3D_MT.py:2136-2142).  All instances of `batch` share
the model (shots of one survey); their lambda/mu/rho buffers are updated in place from
(vp, vs, rho) with mu = rho Vs^2, lambda = rho Vp^2 - 2 mu (:1196-1198).  The backward runs
efm_gradient(EFM_GRAD_EXACT) and the chain rule (efm_chain_rule).
"""
from __future__ import annotations

import torch

from .engine import ShotBatch, chain_rule


class ElasticMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vp, vs, rho, mt, batch: ShotBatch, obs):
        vp = vp.detach().float().contiguous()
        vs = vs.detach().float().contiguous()
        rho = rho.detach().float().contiguous()
        mu = (vs * vs * rho).contiguous()
        lam = (vp * vp * rho - 2.0 * mu).contiguous()
        for i in range(len(batch)):
            batch.set_model(i, lam, mu, rho)
            batch.set_moment_tensor(i, mt.detach().reshape(len(batch), -1, 6)[i].cpu().numpy())
        mod = batch.forward(checkpoints=True)
        res, mis = batch.residual_misfit(mod, obs)
        ctx.batch = batch
        ctx.save_for_backward(vp, vs, rho, res)
        ctx.mt_shape = mt.shape
        return mis.sum()

    @staticmethod
    def backward(ctx, gJ):
        vp, vs, rho, res = ctx.saved_tensors
        batch = ctx.batch
        g, m = batch.gradient(res, exact=True, mt=True)
        n = len(batch)
        acc = torch.zeros((3,) + tuple(vp.shape), dtype=torch.float32, device=vp.device)
        for i in range(n):
            acc += batch.grad_view(g, i)
        gl, gm, gr = acc[0].contiguous(), acc[1].contiguous(), acc[2].contiguous()
        chain_rule(gl, gm, gr, vp, vs, rho)
        nsrc = ctx.mt_shape.numel() // (6 * n)
        gmt = m[:, :nsrc, :].reshape(ctx.mt_shape).to(torch.float32)
        s = gJ.to(torch.float32)
        return s * gl, s * gm, s * gr, s * gmt, None, None


def misfit(vp, vs, rho, mt, batch, obs):
    """Differentiable total misfit (see ElasticMisfit)."""
    return ElasticMisfit.apply(vp, vs, rho, mt, batch, obs)
