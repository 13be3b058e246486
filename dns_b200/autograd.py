"""torch.autograd wrapper of the discrete adjoint (dns_adjoint_energy).

    J = FinalEnergy.apply(u0, nu, dt, nsteps, snapshots)

u0: (3, n, n, n) float64 tensor (any device; moved to the host for the C
ABI), nu: 0-d float64 tensor.  J is main.c's energy after nsteps RK4 steps;
J.backward() fills u0.grad and nu.grad from the hand-written adjoint.
"""
import numpy as np
import torch

from dns_b200 import adjoint_energy


class FinalEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, nu, dt, nsteps, snapshots=20):
        a = u0.detach().cpu().numpy().astype(np.float64)
        J, g, gnu = adjoint_energy(a[0], a[1], a[2], float(nu), float(dt), int(nsteps), int(snapshots))
        ctx.save_for_backward(torch.from_numpy(np.stack(g)).to(u0.device),
                              torch.tensor(gnu, dtype=torch.float64, device=nu.device))
        return torch.tensor(J, dtype=torch.float64, device=u0.device)

    @staticmethod
    def backward(ctx, gJ):
        gu, gnu = ctx.saved_tensors
        return gJ * gu, gJ * gnu, None, None, None
