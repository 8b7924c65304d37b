"""torch.autograd.Function over the forward / backward C-ABI pair.

    traces = receiver_traces(c2q, solver, Q0, dt, nsteps, checkpoint_every)
    loss = ((traces - observed) ** 2).sum() / 2
    loss.backward()            # c2q.grad = dL/d(c^2 at the cubature points)

The solver (a WaveSolver with receivers set) runs the forward on its GPU;
the gradient comes from the hand-written discrete adjoint (bbw_backward),
accumulated in FP64 and returned in c2q's dtype.
"""
import numpy as np
import torch


class ReceiverTraces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, c2q, solver, Q0, dt, nsteps, checkpoint_every):
        solver.set_c2q(c2q.detach().cpu().numpy())
        solver.set_data(np.asarray(Q0, np.float32))
        solver.set_residual(np.zeros(solver.state_size, np.float32))
        solver.set_time(0.0)
        tape = solver.forward(dt, nsteps, checkpoint_every)
        traces = solver.get_traces()
        ctx.solver, ctx.tape, ctx.dtype = solver, tape, c2q.dtype
        return torch.from_numpy(np.ascontiguousarray(traces)).to(c2q.device)

    @staticmethod
    def backward(ctx, g):
        grad = ctx.solver.backward(ctx.tape, g.detach().cpu().numpy())
        ctx.tape.free()
        return (torch.from_numpy(grad).to(device=g.device, dtype=ctx.dtype),
                None, None, None, None, None)


def receiver_traces(c2q, solver, Q0, dt, nsteps, checkpoint_every=50):
    return ReceiverTraces.apply(c2q, solver, Q0, dt, nsteps, checkpoint_every)
