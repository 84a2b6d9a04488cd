"""torch.autograd binding of the discrete adjoint (dtmx_forward_adjoint).

flux_objective(eps, make_sim, lo, nsteps, plane_x, omega) returns the Poynting
flux J of the running DFT at omega through the plane x = plane_x after
nsteps, as a differentiable function of the per-node permittivity eps
(shape (3, n0, n1, n2), the three E components over the design box starting
at cell lo).  The forward call runs the simulation and the adjoint once and
keeps dJ/d eps; backward scales it by the incoming gradient.  make_sim()
must return a fresh Simulation (state at t = 0) with its materials and
sources set.
"""
import numpy as np
import torch


class FluxObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eps, make_sim, lo, nsteps, plane_x, omega, checkpoint_every):
        sim = make_sim()
        try:
            sim.set_design(lo, eps.detach().to("cpu", torch.float32).numpy())
            J, grad = sim.forward_adjoint(nsteps, plane_x, omega, checkpoint_every)
        finally:
            sim.close()
        ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(grad)).to(eps.device, eps.dtype))
        return eps.new_tensor(J)

    @staticmethod
    def backward(ctx, gJ):
        (grad,) = ctx.saved_tensors
        return gJ * grad, None, None, None, None, None, None


def flux_objective(eps, make_sim, lo, nsteps, plane_x, omega, checkpoint_every=100):
    return FluxObjective.apply(eps, make_sim, tuple(lo), int(nsteps), int(plane_x), float(omega), int(checkpoint_every))
