"""torch.autograd binding of the solver's hand-written adjoint (kami_vbd_backward).

``StrandStiffnessRollout`` maps per-strand bend/twist stiffness scales to the positions after a
rollout of ``frames`` steps.  The rest Darboux quaternions, whose magnitude is the bend/twist
stiffness (Sim::setYoung, YarnBall/YBSimulator.cu:300-320), are  qRest_i = scale[strand(i)] *
unit_i.

Checkpointing.  The forward pass keeps a device checkpoint of the full state every
``checkpoint_every`` steps, and the rollout falls into segments of that many steps.  A recorded step
costs (num_itr + 1) * 32 + 48 B of tape per slot and substep.  The last segments of the rollout, as
many as ``tape_budget_bytes`` holds, are recorded during the forward pass itself (kami_vbd_step_record
instead of kami_vbd_step), so the backward pass differentiates them straight away; every earlier
segment is recomputed in the backward pass from its checkpoint: restore, record its steps, run the
adjoint back to the checkpoint.  With a budget of 0 every segment is recomputed (the least memory);
the default (None) allows a quarter of the device memory that is free when the forward pass starts.
The tape lives in the solver handle, so run the backward pass of a rollout before the next rollout
on the same solver records; if another rollout recorded in between, the backward pass recomputes
every segment from the checkpoints instead.

With ``tiles_per_chunk`` the backward pass works on one window of warp tiles at a time (strands are
independent; the window is rounded up to whole groups of tiles when strands run across several), so
the tape memory is bounded by the window; every segment is then recomputed, and each window restores
its checkpoints and moves its adjoints for its own strands only.  ``body_transforms``
((frames, 7): rotation x y z w, translation per frame) moves the body SDF frame by frame, in the
forward pass and in the recorded steps alike.  The solver must use the fused form with the colour2
schedule (wind is allowed); a frame of several substeps (dt > max_h) is recorded substep by substep.
"""
from __future__ import annotations

import itertools

import torch

_rollout_ids = itertools.count(1)


def _segments_recorded_in_forward(solver, frames, dt, k, tiles_per_chunk, budget, device):
    """Number of trailing segments whose tape fits the budget (0 with tile windows)."""
    tiles = solver.tile_count()
    if 0 < tiles_per_chunk < tiles:
        return 0
    nseg = -(-frames // k)
    per_seg = solver.tape_bytes_per_substep() * solver.substeps(dt) * k
    if budget is None:
        budget = torch.cuda.mem_get_info(device)[0] // 4
    return int(min(nseg, budget // per_seg)) if per_seg > 0 else 0


class StrandStiffnessRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, scale, solver, unit, strand_of, init_state, frames, dt, checkpoint_every, tiles_per_chunk=0,
                body_transforms=None, tape_budget_bytes=None):
        """scale: (S,) CUDA float32; unit: (V, 4) CUDA rest Darboux at scale 1; strand_of: (V,) long;
        init_state: flat CUDA float32 state (Solver.get_state_into layout).  Returns (V, 3) positions."""
        k = max(1, int(checkpoint_every))
        nseg = -(-frames // k)
        m = _segments_recorded_in_forward(solver, frames, dt, k, int(tiles_per_chunk), tape_budget_bytes,
                                          init_state.device)
        first_recorded = nseg - m  # segments >= this one are recorded in the forward pass
        qr = (unit * scale[strand_of][:, None]).contiguous()
        torch.cuda.synchronize()
        solver.set_rest_darboux(qr)
        solver.set_state_from(init_state)
        rid = next(_rollout_ids)
        if m > 0:
            solver.tape_reserve(m * k * solver.substeps(dt), 0)
            solver._tape_rollout = rid
        ckpts = []
        for f in range(frames):
            seg = f // k
            if f % k == 0:
                ckpts.append(solver.get_state_into(torch.empty_like(init_state)))
            _move_body(solver, body_transforms, f)
            if seg >= first_recorded:
                solver.step_record(dt)
            else:
                solver.step(dt)
        x = torch.empty((solver.num_vertices, 3), dtype=torch.float32, device=init_state.device)
        solver.get_positions_velocities(x, None)
        ctx.solver, ctx.ckpts, ctx.frames, ctx.dt, ctx.k = solver, ckpts, frames, dt, k
        ctx.chunk = int(tiles_per_chunk)
        ctx.body = body_transforms
        ctx.recorded, ctx.rid = m, rid
        ctx.save_for_backward(unit, strand_of, scale)
        return x

    @staticmethod
    def backward(ctx, gx):
        unit, strand_of, scale = ctx.saved_tensors
        solver, k = ctx.solver, ctx.k
        nv = solver.num_vertices
        dev = gx.device
        ax = gx.detach().to(torch.float32).contiguous().clone()
        av = torch.zeros((nv, 3), dtype=torch.float32, device=dev)
        avl = torch.zeros_like(av)
        aq = torch.zeros((nv, 4), dtype=torch.float32, device=dev)
        nseg = len(ctx.ckpts)
        m = ctx.recorded if solver._tape_rollout == ctx.rid else 0
        solver._tape_rollout = None  # this pass consumes the tape or reallocates it
        # the rest Darboux of this rollout (another rollout on the solver may have set its own since)
        solver.set_rest_darboux((unit * scale[strand_of][:, None]).contiguous())
        if m > 0:  # the tail recorded in the forward pass, then the rest recomputed from checkpoints
            solver.zero_rest_darboux_grad()
            torch.cuda.synchronize()
            solver.backward(ax, av, avl, aq)
            for seg in reversed(range(nseg - m)):
                _recompute_segment(ctx, solver, seg)
                solver.backward(ax, av, avl, aq)
        else:
            tiles = solver.tile_count()
            chunk = ctx.chunk if 0 < ctx.chunk < tiles else tiles
            group = solver.tiles_per_group()  # tape windows are whole groups of tiles
            chunk = min(tiles, -(-chunk // group) * group)
            solver.tape_reserve(k * solver.substeps(ctx.dt), chunk)  # one tape entry per substep
            solver.zero_rest_darboux_grad()
            torch.cuda.synchronize()
            for t0 in range(0, tiles, chunk):
                solver.set_tape_window(t0, min(tiles, t0 + chunk))
                for seg in reversed(range(nseg)):
                    _recompute_segment(ctx, solver, seg)
                    solver.backward(ax, av, avl, aq)
        gqr = torch.empty((nv, 4), dtype=torch.float32, device=dev)
        solver.get_rest_darboux_grad(gqr)
        per_vertex = (gqr * unit).sum(-1)
        gscale = torch.zeros_like(scale).index_add_(0, strand_of, per_vertex)
        return gscale, None, None, None, None, None, None, None, None, None, None


def _recompute_segment(ctx, solver, seg):
    solver.restore_tape_window_from(ctx.ckpts[seg])  # the window's strands (all of them without a window)
    n = min(ctx.k, ctx.frames - seg * ctx.k)
    for j in range(n):
        _move_body(solver, ctx.body, seg * ctx.k + j)
        solver.step_record(ctx.dt)


def _move_body(solver, body_transforms, frame):
    if body_transforms is not None:
        solver.set_body_transform(body_transforms[frame][:4], body_transforms[frame][4:7])


def rollout_positions(scale, solver, unit, strand_of, init_state, frames, dt, checkpoint_every=10, tiles_per_chunk=0,
                      body_transforms=None, tape_budget_bytes=None):
    return StrandStiffnessRollout.apply(scale, solver, unit, strand_of, init_state, frames, dt, checkpoint_every,
                                        tiles_per_chunk, body_transforms, tape_budget_bytes)
