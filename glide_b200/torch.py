"""PyTorch boundary (mirror of glide/torch.py:4-59).

`GlideStep.apply(t, dt, model, level, H_prev, bed, beta, smb)` runs one
forward step on hierarchy level `level` and returns new tensors (u, v, H);
its backward solves the adjoint system and returns the gradients for
(H_prev, bed, beta, smb).  The forward state (u, v, H, mask, phi) is
checkpointed in `ctx` per step and restored before the adjoint solve, so a
sequence of steps can be differentiated with torch.autograd.
"""
from __future__ import annotations

import torch


class GlideStep(torch.autograd.Function):

    @staticmethod
    def forward(ctx, t, dt, model, level, H_prev, bed, beta, smb):
        ctx.t, ctx.dt, ctx.model, ctx.level = t, dt, model, level
        model.set_top_level(level)
        mg = model.mg
        mg.state.H_prev.set(H_prev.detach(), start_level=level)
        mg.state.H.set(H_prev.detach(), start_level=level)
        mg.geometry.bed.set(bed.detach(), start_level=level)
        mg.sliding.beta.set(beta.detach(), start_level=level)
        mg.forcing.smb.set(smb.detach(), start_level=level)
        model.forward(t, dt, update_geometry=False)
        lev = mg[level].state
        out_dtype = H_prev.dtype
        u = lev.u.data.to(out_dtype).clone()
        v = lev.v.data.to(out_dtype).clone()
        H = lev.H.data.to(out_dtype).clone()
        mask = lev.mask.data.clone()
        phi = lev.phi.data.clone()
        ctx.save_for_backward(u, v, H, mask, phi, H_prev, bed, beta, smb)
        return u, v, H

    @staticmethod
    def backward(ctx, gu, gv, gH):
        t, dt, model, level = ctx.t, ctx.dt, ctx.model, ctx.level
        u, v, H, mask, phi, H_prev, bed, beta, smb = ctx.saved_tensors
        mg = model.mg
        model.set_top_level(level)
        mg.state.H_prev.set(H_prev.detach(), start_level=level)
        mg.geometry.bed.set(bed.detach(), start_level=level)
        mg.sliding.beta.set(beta.detach(), start_level=level)
        mg.forcing.smb.set(smb.detach(), start_level=level)
        mg.state.u.set(u, start_level=level)
        mg.state.v.set(v, start_level=level)
        mg.state.H.set(H, start_level=level)
        mg.state.phi.set(phi, start_level=level)
        mg.state.mask.set(mask, start_level=level)
        zero = lambda g, ref: torch.zeros_like(ref) if g is None else g
        model.backward(t, dt, dJdu=zero(gu, u), dJdv=zero(gv, v), dJdH=zero(gH, H))
        lv = mg[level]
        dt_ = H_prev.dtype
        return (None, None, None, None,
                lv.state.H_prev.grad.to(dt_).clone(), lv.geometry.bed.grad.to(dt_).clone(),
                lv.sliding.beta.grad.to(dt_).clone(), lv.forcing.smb.grad.to(dt_).clone())
