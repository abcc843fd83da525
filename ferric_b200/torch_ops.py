"""``torch.autograd.Function`` wrapper of the RI-MP2 energy and its adjoint.

``RiMp2Energy.apply(b_ov, eps_occ, eps_vir, precision)`` returns the closed-shell
MP2 correlation energy ``E = E_os + E_ss`` as a 0-d float64 tensor.  Its
backward gives ``dE/dB = Gamma`` (``4 x_ov`` of ferric-mp2/src/zvector.rs:651-703),
``dE/d eps_occ`` and ``dE/d eps_vir`` (``2 diag(P)``, ferric-mp2/src/oo_rimp2.rs:1170-1300).

When any input requires grad, forward runs the fused energy+adjoint kernels
once (pair blocks recomputed, never stored) and keeps Gamma for backward;
otherwise it runs the energy-only kernel.
"""
from __future__ import annotations

import torch

from .rimp2 import rimp2_energy, rimp2_energy_grad


class RiMp2Energy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, b_ov, eps_occ, eps_vir, precision="f64"):
        if not b_ov.is_cuda:
            raise ValueError("RiMp2Energy: inputs must be CUDA tensors")
        b = b_ov.detach().to(torch.float64).contiguous()
        o = eps_occ.detach().to(torch.float64).contiguous()
        v = eps_vir.detach().to(torch.float64).contiguous()
        if any(ctx.needs_input_grad[:3]):
            sc, gamma, d_o, d_v = rimp2_energy_grad(b, o, v, precision)
            ctx.save_for_backward(gamma, d_o, d_v)
            e_os, e_ss = sc.e_os, sc.e_ss
        else:
            e_os, e_ss = rimp2_energy(b, o, v, precision=precision)
        ctx.spin = (e_os, e_ss)
        return torch.tensor(e_os + e_ss, dtype=torch.float64, device=b.device)

    @staticmethod
    def backward(ctx, g):
        gamma, d_o, d_v = ctx.saved_tensors
        gb = go = gv = None
        if ctx.needs_input_grad[0]:
            gb = gamma * g
        if ctx.needs_input_grad[1]:
            go = d_o * g
        if ctx.needs_input_grad[2]:
            gv = d_v * g
        return gb, go, gv, None


def rimp2_energy_autograd(b_ov, eps_occ, eps_vir, precision="f64"):
    return RiMp2Energy.apply(b_ov, eps_occ, eps_vir, precision)
