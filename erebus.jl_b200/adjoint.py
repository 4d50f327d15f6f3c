"""Gradients of the heat path from Python.

`heat_gradient` runs erebus_adjoint_heat: n timesteps forward on the GPU,
the objective J (mean of the 4-P-node average of tk2 over the basic nodes
inside the body after the last step) and, by the reverse sweep, dJ/dphim per
marker and dJ/d(26Al/27Al).  `HeatObjective` wraps it as a
torch.autograd.Function, the counterpart of the ChainRulesCore rrule a Julia
binding defines for the same call.  The adjoint covers states at mechanical
rest (`at_rest`); other states raise ErebusError (EINVAL).
"""
import torch

from .device import Simulation


def at_rest(st):
    """Puts a HostState at mechanical rest: no self-gravity, no boundary
    strain rate, reactions and subgrid diffusion off, zero marker stresses.
    Velocities, porosity change and marker motion then vanish and the heat
    path carries the whole dependence of J on porosity and 26Al/27Al."""
    p = st.p
    p.G = 0.0
    p.strainrate = 0.0
    p.reaction_active = 0
    p.dsubgrids = 0.0
    p.dsubgridt = 0.0
    st.m["sxxm"][:] = 0.0
    st.m["sxym"][:] = 0.0
    return st


def heat_gradient(host, n_steps, checkpoint_every=5, first_timestep=1):
    """(J, dJ/dphim, dJ/dratio_al, ErebusAdjointStats) of n_steps timesteps
    from HostState `host` (which is not modified)."""
    sim = Simulation(host)
    try:
        return sim.adjoint_heat(n_steps, checkpoint_every, first_timestep)
    finally:
        sim.close()


class HeatObjective(torch.autograd.Function):
    """J(phim, ratio_al) with the adjoint as its backward.

    forward(phim, ratio_al, host, n_steps, checkpoint_every): `phim` is a
    float64 tensor of the host's marknum porosities, `ratio_al` a scalar
    tensor; `host` supplies everything else (it is copied, not modified)."""

    @staticmethod
    def forward(ctx, phim, ratio_al, host, n_steps, checkpoint_every=5):
        st = host.copy()
        st.p = type(host.p).from_buffer_copy(host.p)
        n = st.marknum
        phi = phim.detach().to("cpu", torch.float64).numpy()
        st.m["phim"][:n] = phi
        st.m["phinewm"][:n] = phi
        st.p.ratio_al = float(ratio_al)
        J, g, gr, _ = heat_gradient(st, n_steps, checkpoint_every)
        ctx.save_for_backward(torch.from_numpy(g).to(phim.device, phim.dtype),
                              torch.tensor(gr, dtype=phim.dtype, device=phim.device))
        return torch.tensor(J, dtype=phim.dtype, device=phim.device)

    @staticmethod
    def backward(ctx, gJ):
        g, gr = ctx.saved_tensors
        return gJ * g, gJ * gr, None, None, None
