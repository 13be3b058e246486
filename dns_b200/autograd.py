"""torch.autograd wrapper of the discrete adjoint (dns_adjoint_energy).

    J = FinalEnergy.apply(u0, nu, dt, nsteps, snapshots, precision)

u0: (3, n, n, n) float64 tensor (any device; moved to the host for the C
ABI), nu: 0-d float64 tensor.  J is main.c's energy after nsteps RK4 steps.
The forward call runs the forward sweep only; J.backward() runs the
hand-written adjoint (forward sweep with checkpoints, reverse sweep) and
fills u0.grad and nu.grad.  precision: DNS_PREC_FP64 (default) or
DNS_PREC_MIXED.
"""
import numpy as np
import torch

from dns_b200 import DNS_PREC_FP64, adjoint_energy, final_energy


class FinalEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, nu, dt, nsteps, snapshots=20, precision=DNS_PREC_FP64):
        a = u0.detach().cpu().numpy().astype(np.float64)
        J = final_energy(a[0], a[1], a[2], float(nu), float(dt), int(nsteps), int(precision))
        ctx.save_for_backward(u0.detach(), nu.detach())
        ctx.cfg = (float(dt), int(nsteps), int(snapshots), int(precision))
        return torch.tensor(J, dtype=torch.float64, device=u0.device)

    @staticmethod
    def backward(ctx, gJ):
        u0, nu = ctx.saved_tensors
        dt, nsteps, snapshots, precision = ctx.cfg
        a = u0.cpu().numpy().astype(np.float64)
        _, g, gnu = adjoint_energy(a[0], a[1], a[2], float(nu), dt, nsteps, snapshots, precision)
        gu = torch.from_numpy(np.stack(g)).to(u0.device)
        gn = torch.tensor(gnu, dtype=torch.float64, device=nu.device)
        return gJ * gu, gJ * gn, None, None, None, None
