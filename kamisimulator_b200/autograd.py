"""torch.autograd binding of the solver's hand-written adjoint (kami_vbd_backward).

``StrandStiffnessRollout`` maps per-strand bend/twist stiffness scales to the positions after a
rollout of ``frames`` steps.  The rest Darboux quaternions, whose magnitude is the bend/twist
stiffness (Sim::setYoung, YarnBall/YBSimulator.cu:300-320), are  qRest_i = scale[strand(i)] *
unit_i.  The forward pass keeps a device checkpoint of the full state every ``checkpoint_every``
steps.  The backward pass walks the segments in reverse: it restores the segment's checkpoint,
records its steps, and runs the adjoint back to the checkpoint.  With ``tiles_per_chunk`` it does so
for one window of warp tiles at a time (strands are independent; the window is rounded up to whole
groups of tiles when strands run across several), so the tape memory is bounded by
the window: (num_itr + 1) * 32 + 48 B per slot and recorded step.  ``body_transforms`` ((frames, 7):
rotation x y z w, translation per frame) moves the body SDF frame by frame, in the forward pass and
in the recorded steps alike.  The solver must use the fused form with the colour2 schedule (wind is
allowed); a frame of several substeps (dt > max_h) is recorded substep by substep.
"""
from __future__ import annotations

import torch


class StrandStiffnessRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, scale, solver, unit, strand_of, init_state, frames, dt, checkpoint_every, tiles_per_chunk=0,
                body_transforms=None):
        """scale: (S,) CUDA float32; unit: (V, 4) CUDA rest Darboux at scale 1; strand_of: (V,) long;
        init_state: flat CUDA float32 state (Solver.get_state_into layout).  Returns (V, 3) positions."""
        k = max(1, int(checkpoint_every))
        qr = (unit * scale[strand_of][:, None]).contiguous()
        torch.cuda.synchronize()
        solver.set_rest_darboux(qr)
        solver.set_state_from(init_state)
        ckpts = []
        for f in range(frames):
            if f % k == 0:
                ckpts.append(solver.get_state_into(torch.empty_like(init_state)))
            _move_body(solver, body_transforms, f)
            solver.step(dt)
        x = torch.empty((solver.num_vertices, 3), dtype=torch.float32, device=init_state.device)
        solver.get_positions_velocities(x, None)
        ctx.solver, ctx.ckpts, ctx.frames, ctx.dt, ctx.k = solver, ckpts, frames, dt, k
        ctx.chunk = int(tiles_per_chunk)
        ctx.body = body_transforms
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
        tiles = solver.tile_count()
        chunk = ctx.chunk if 0 < ctx.chunk < tiles else tiles
        group = solver.tiles_per_group()  # tape windows are whole groups of tiles
        chunk = min(tiles, -(-chunk // group) * group)
        solver.tape_reserve(k * solver.substeps(ctx.dt), chunk)  # one tape entry per substep
        solver.zero_rest_darboux_grad()
        torch.cuda.synchronize()
        for t0 in range(0, tiles, chunk):
            solver.set_tape_window(t0, min(tiles, t0 + chunk))
            for seg in reversed(range(len(ctx.ckpts))):
                solver.set_state_from(ctx.ckpts[seg])
                n = min(k, ctx.frames - seg * k)
                for j in range(n):
                    _move_body(solver, ctx.body, seg * k + j)
                    solver.step_record(ctx.dt)
                solver.backward(ax, av, avl, aq)
        gqr = torch.empty((nv, 4), dtype=torch.float32, device=dev)
        solver.get_rest_darboux_grad(gqr)
        per_vertex = (gqr * unit).sum(-1)
        gscale = torch.zeros_like(scale).index_add_(0, strand_of, per_vertex)
        return gscale, None, None, None, None, None, None, None, None, None


def _move_body(solver, body_transforms, frame):
    if body_transforms is not None:
        solver.set_body_transform(body_transforms[frame][:4], body_transforms[frame][4:7])


def rollout_positions(scale, solver, unit, strand_of, init_state, frames, dt, checkpoint_every=10, tiles_per_chunk=0,
                      body_transforms=None):
    return StrandStiffnessRollout.apply(scale, solver, unit, strand_of, init_state, frames, dt, checkpoint_every,
                                        tiles_per_chunk, body_transforms)
