"""PyTorch boundary (mirror of glide/torch.py:4-59).

`GlideStep.apply(t, dt, model, level, H_prev, bed, beta, smb)` runs one
forward step on hierarchy level `level` and returns new tensors (u, v, H);
its backward solves the adjoint system and returns the gradients for
(H_prev, bed, beta, smb).  The forward state (u, v, H, mask, phi) of each step
is what the adjoint solve linearises about.  The reference keeps it for every
step (glide/torch.py:29), and so does this module by default.

With `checkpointing(model, every=k)` a chain of steps keeps the solved state
of every k-th step only.  The backward pass of a step whose state was dropped
re-solves the steps since the last kept state, each from the previous step's
solution exactly as the forward pass ran them, and holds that segment until
its steps have been differentiated.  The recomputed states are bit-identical
to the dropped ones, so are the gradients.  Peak memory falls from one state
per step to one per k steps plus one segment; the cost is at most one extra
forward solve per step.
"""
from __future__ import annotations

import math

import torch


def _state_bytes(model, level):
    lev = model.mg[level].state
    return sum(t.numel() * t.element_size() for t in (lev.u.data, lev.v.data, lev.H.data, lev.mask.data,
                                                        lev.phi.data))


class Checkpointing:
    """Which solved states of a chain of GlideSteps on one model are kept for
    backward (no counterpart in the reference, which keeps all of them).

    every: keep the state of every `every`-th step of the chain (the first
    step of a chain is always a segment start).  Steps of a chain must follow
    one another on the model -- each step warm-starts from the solution the
    previous one left -- as in a time loop.  A step before which the model's
    handle launched any other kernel (another solve, a field set outside
    GlideStep), or which runs on another level, starts a new segment and
    stores its starting state, so recomputation never relies on a state it
    cannot reproduce.  Writing the model's state arrays through tensor views
    between two steps of a chain is not detected and must not be done.
    """

    def __init__(self, every: int = 1):
        if int(every) < 1:
            raise ValueError("every must be >= 1")
        self.every = int(every)
        self._next_id = 0
        self._chain_pos = 0       # position of the next step in its chain
        self._last = None         # (launch count, level, record) at the end of the last recorded forward
        self._segment = {}        # recomputed states of the segment being differentiated
        self.recomputed_steps = 0  # forward solves run again by backward passes
        self.kept_steps = 0
        self.dropped_steps = 0

    @staticmethod
    def interval_for(max_bytes: float, n_steps: int, state_bytes: float) -> int:
        """The smallest interval whose kept states plus one recomputed
        segment, (ceil(n_steps / k) + k) state_bytes, fit in max_bytes."""
        for k in range(1, n_steps + 1):
            if (math.ceil(n_steps / k) + k) * state_bytes <= max_bytes:
                return k
        raise ValueError(f"{n_steps} steps of {state_bytes:.3g} B states do not fit in {max_bytes:.3g} B "
                         "even with recomputation")


class _Record:
    __slots__ = ("id", "t", "dt", "level", "inputs", "entry", "state", "prev")

    def __init__(self, rid, t, dt, level, inputs):
        self.id, self.t, self.dt, self.level, self.inputs = rid, t, dt, level, inputs
        self.entry = None   # (u, v, mask, phi) before the step, for a segment start
        self.state = None   # (u, v, H, mask, phi) after the step, when kept
        self.prev = None    # the previous record of the chain


def checkpointing(model, every: int | None = None, max_bytes: float | None = None, n_steps: int | None = None,
                  level: int = 0):
    """Set the GlideStep memory policy of `model` and return it.

    every = 1 (or no argument) keeps every step's state, as the reference
    does.  Alternatively max_bytes and n_steps pick the interval: the
    smallest whose kept states plus one recomputed segment fit in max_bytes
    (state size taken at `level`)."""
    if every is None:
        if max_bytes is None:
            every = 1
        else:
            if n_steps is None:
                raise ValueError("max_bytes needs n_steps")
            every = Checkpointing.interval_for(max_bytes, n_steps, _state_bytes(model, level))
    policy = Checkpointing(every)
    model._glide_checkpointing = policy
    return policy


def _policy(model):
    return getattr(model, "_glide_checkpointing", None)


def _snapshot(lev, with_H):
    names = ("u", "v", "H", "mask", "phi") if with_H else ("u", "v", "mask", "phi")
    return tuple(getattr(lev, n).data.detach().clone() for n in names)


def _set_inputs(mg, level, H_prev, bed, beta, smb):
    mg.state.H_prev.set(H_prev, start_level=level)
    mg.state.H.set(H_prev, start_level=level)
    mg.geometry.bed.set(bed, start_level=level)
    mg.sliding.beta.set(beta, start_level=level)
    mg.forcing.smb.set(smb, start_level=level)


def _set_state(mg, level, u, v, mask, phi, H=None):
    mg.state.u.set(u, start_level=level)
    mg.state.v.set(v, start_level=level)
    if H is not None:
        mg.state.H.set(H, start_level=level)
    mg.state.phi.set(phi, start_level=level)
    mg.state.mask.set(mask, start_level=level)


def _solved_state(model, policy, rec):
    """(u, v, H, mask, phi) after the step of `rec`: kept, from the segment
    being differentiated, or recomputed from the last kept state."""
    if rec.state is not None:
        return rec.state
    if rec.id in policy._segment:
        return policy._segment.pop(rec.id)
    # walk back to the segment start: a stored starting state, or the step
    # after a kept state
    chain = [rec]
    while True:
        r = chain[-1]
        if r.entry is not None:
            warm = r.entry
            break
        if r.prev is None:
            raise RuntimeError("GlideStep checkpointing: no kept state to recompute this step from")
        if r.prev.state is not None:
            warm = r.prev.state[:2] + r.prev.state[3:]
            break
        chain.append(r.prev)
    mg = model.mg
    out = None
    for r in reversed(chain):
        u, v, mask, phi = warm
        model.set_top_level(r.level)
        _set_state(mg, r.level, u, v, mask, phi)
        _set_inputs(mg, r.level, *r.inputs)
        model.forward_solver.solve(r.dt, start_level=r.level)  # no post-forward hooks
        out = _snapshot(mg[r.level].state, True)
        policy.recomputed_steps += 1
        if r is not rec:
            policy._segment[r.id] = out
        warm = out[:2] + out[3:]
    return out


class GlideStep(torch.autograd.Function):

    @staticmethod
    def forward(ctx, t, dt, model, level, H_prev, bed, beta, smb):
        ctx.t, ctx.dt, ctx.model, ctx.level = t, dt, model, level
        model.set_top_level(level)
        mg = model.mg
        policy = _policy(model)
        rec = None
        if policy is not None and policy.every > 1 and any(ctx.needs_input_grad):
            h = mg.hierarchy
            rec = _Record(policy._next_id, t, dt, level,
                          tuple(x.detach() for x in (H_prev, bed, beta, smb)))
            policy._next_id += 1
            last = policy._last
            follows = last is not None and last[0] == h.launch_count() and last[1] == level
            if follows:
                rec.prev = last[2]
                policy._chain_pos += 1
            else:
                policy._chain_pos = 0
                rec.entry = _snapshot(mg[level].state, False)  # the warm start of a new segment
        _set_inputs(mg, level, *(x.detach() for x in (H_prev, bed, beta, smb)))
        model.forward(t, dt, update_geometry=False)
        lev = mg[level].state
        out_dtype = H_prev.dtype
        u = lev.u.data.to(out_dtype).clone()
        v = lev.v.data.to(out_dtype).clone()
        H = lev.H.data.to(out_dtype).clone()
        if rec is None:
            ctx.save_for_backward(u, v, H, lev.mask.data.clone(), lev.phi.data.clone(), H_prev, bed, beta, smb)
            ctx.rec = None
            return u, v, H
        keep = policy._chain_pos % policy.every == 0
        if keep:
            if out_dtype == lev.u.data.dtype:
                rec.state = (u, v, H, lev.mask.data.clone(), lev.phi.data.clone())
            else:
                rec.state = _snapshot(lev, True)
            policy.kept_steps += 1
        else:
            policy.dropped_steps += 1
        policy._last = (mg.hierarchy.launch_count(), level, rec)
        ctx.rec = rec
        ctx.save_for_backward(H_prev, bed, beta, smb)
        return u, v, H

    @staticmethod
    def backward(ctx, gu, gv, gH):
        t, dt, model, level = ctx.t, ctx.dt, ctx.model, ctx.level
        mg = model.mg
        rec = ctx.rec
        if rec is None:
            u, v, H, mask, phi, H_prev, bed, beta, smb = ctx.saved_tensors
        else:
            H_prev, bed, beta, smb = ctx.saved_tensors
            policy = _policy(model)
            u, v, H, mask, phi = _solved_state(model, policy, rec)
            policy._last = None  # recomputation moved the handle: the next forward starts a new segment
        model.set_top_level(level)
        mg.state.H_prev.set(H_prev.detach(), start_level=level)
        mg.geometry.bed.set(bed.detach(), start_level=level)
        mg.sliding.beta.set(beta.detach(), start_level=level)
        mg.forcing.smb.set(smb.detach(), start_level=level)
        _set_state(mg, level, u, v, mask, phi, H=H)
        zero = lambda g, ref: torch.zeros_like(ref) if g is None else g
        model.backward(t, dt, dJdu=zero(gu, u), dJdv=zero(gv, v), dJdH=zero(gH, H))
        lv = mg[level]
        dt_ = H_prev.dtype
        if rec is not None:
            rec.inputs = rec.entry = rec.state = None  # this step's backward is done
        return (None, None, None, None,
                lv.state.H_prev.grad.to(dt_).clone(), lv.geometry.bed.grad.to(dt_).clone(),
                lv.sliding.beta.grad.to(dt_).clone(), lv.forcing.smb.grad.to(dt_).clone())
