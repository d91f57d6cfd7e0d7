"""A time step as a torch.autograd.Function (test harness).

StepFunction runs one step forward and, in backward, the step's adjoint.
Here the step is oracle/adjoint64.Step64 (the FP64 oracle's step and the
FP64 reference adjoint); an objective written with torch operations on the
returned state then gets its gradients with respect to the initial state,
the inflow profile and the drag scale from loss.backward().
"""
import numpy as np
import torch

from oracle import adjoint64


class StepFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, step, n, wp, drag, *state):
        step.drag = None if drag is None else drag.detach().numpy().copy()
        st = {k: t.detach().numpy() for k, t in zip(adjoint64.STATE, state)}
        out, tape = step.forward(n, st, wp.detach().numpy())
        ctx.step, ctx.n, ctx.tape, ctx.wp = step, n, tape, wp.detach().numpy().copy()
        ctx.drag = step.drag
        ctx.has_drag = drag is not None
        return tuple(torch.from_numpy(np.ascontiguousarray(out[k])) for k in adjoint64.STATE)

    @staticmethod
    def backward(ctx, *grads):
        seeds = {k: g.numpy() for k, g in zip(adjoint64.STATE, grads)}  # unused outputs come as zeros
        ctx.step.drag = ctx.drag
        b, pg = ctx.step.adjoint(ctx.n, ctx.tape, ctx.wp, seeds)
        dg = torch.from_numpy(pg["drag"]) if ctx.has_drag else None
        return (None, None, torch.from_numpy(pg["wp"]), dg,
                *[torch.from_numpy(np.ascontiguousarray(b[k])) for k in adjoint64.STATE])


def tke_torch(ip, jp, kp, state, box):
    """adjoint64.tke written with torch operations on the state tensors."""
    (i0, i1), (j0, j1), (k0, k1) = box
    lo = {n: [adjoint64.FL._ev(b.split(":")[0], ip, jp, kp) for b in adjoint64.FL._BOUNDS[n]] for n in "uvw"}

    def view(n, a, b, c):
        t, (li, lj, lk) = state[n], lo[n]
        return t[a[0] - li:a[1] - li + 1, b[0] - lj:b[1] - lj + 1, c[0] - lk:c[1] - lk + 1]

    I, J, K = (i0, i1), (j0, j1), (k0, k1)
    sh = lambda r: (r[0] - 1, r[1] - 1)
    uc = 0.5 * (view("u", sh(I), J, K) + view("u", I, J, K))
    vc = 0.5 * (view("v", I, sh(J), K) + view("v", I, J, K))
    wc = 0.5 * (view("w", I, J, sh(K)) + view("w", I, J, K))
    return torch.mean(0.5 * (uc * uc + vc * vc + wc * wc))


class TkeObjective(torch.autograd.Function):
    """The config-3 objective on the GPU through the C ABI: J(wp, drag) =
    time-mean resolved TKE of a box over nt steps from the state in slot
    `init` of a GpuAdjoint.  forward runs the CUDA steps keeping a checkpoint
    every ckpt steps (les_halo_b200.tke_forward); backward runs the device
    step adjoint over the checkpoints with recomputation
    (les_halo_b200.tke_reverse) and returns the gradients of the inflow
    profile wp(jp, kp) and the drag scale s(ip, jp)."""

    @staticmethod
    def forward(ctx, wp, drag, gpu, adj, init, n0, nt, box, ckpt):
        import les_halo_b200 as lh
        adj.load(init)
        gpu.set_wind_profile(np.asfortranarray(wp.detach().numpy(), dtype=np.float32))
        lh.set_drag(gpu, drag.detach().numpy())
        J = lh.tke_forward(gpu, adj, n0, nt, box, ckpt)
        ctx.args = (gpu, adj, n0, nt, box, ckpt)
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        import les_halo_b200 as lh
        g = lh.tke_reverse(*ctx.args)
        return (gJ * torch.from_numpy(g["wp"]), gJ * torch.from_numpy(g["drag"]),
                None, None, None, None, None, None, None)
