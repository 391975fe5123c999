"""torch.autograd wrappers of the SF-CIS(D) and EE-CPS(D-3) energies (the
backward pass only).

`cisd_energies(s, tensors, symR, nroot)` returns the SF-CIS energies w0 and
second-order corrections w^(2) of the roots of irrep symR as differentiable
functions of the spin-free DPD integrals (ijka, abij, iabj, abci) and Eorb.
The forward pass is cpsd_cisd_energies, the backward pass
cpsd_cisd_gradient (a hand-written adjoint on the device); torch holds the
tensors and the graph only.  ijkl and abcd do not enter these energies.

`cpsd3_energies(s, tensors, symR, nroot)` adds the third-order corrections
w^(3) (cpsd_cpsd3_energies / cpsd_cpsd3_gradient), which read all six lists.
"""
import numpy as np
import torch

from . import api

KEYS = ("ijka", "abij", "iabj", "abci", "eorb")


class CisdEnergies(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ijka, abij, iabj, abci, eorb, s, sysc, par, symR, nroot):
        t = dict(zip(KEYS, (ijka, abij, iabj, abci, eorb)))
        st = api.integrals_struct(t)
        w0, w2, L = api.cisd_energies(s, sysc, st, par, symR, nroot)
        ctx.save_for_backward(ijka, abij, iabj, abci, eorb, L)
        ctx.meta = (sysc, par, symR, w0)
        return torch.from_numpy(w0), torch.from_numpy(w2)

    @staticmethod
    def backward(ctx, g0, g2):
        ijka, abij, iabj, abci, eorb, L = ctx.saved_tensors
        sysc, par, symR, w0 = ctx.meta
        n = len(w0)
        g0 = np.zeros(n) if g0 is None else g0.detach().cpu().double().numpy()
        g2 = np.zeros(n) if g2 is None else g2.detach().cpu().double().numpy()
        t = dict(zip(KEYS, (ijka, abij, iabj, abci, eorb)))
        grads = {k: torch.zeros_like(v) for k, v in t.items()}
        api.cisd_gradient(sysc, api.integrals_struct(t), par, symR, w0, L, g0, g2, grads)
        return tuple(grads[k] for k in KEYS) + (None,) * 5


def cisd_energies(s, tensors, symR, nroot, **params):
    """(w0, w2) of nroot roots of irrep symR; tensors: dict of float64 CUDA
    tensors with keys ijka, abij, iabj, abci, eorb (requires_grad as needed);
    params: cpsd_params fields (davidson_conv, diis_max_err, ...)."""
    sysc = api.make_system(s)
    par = api.make_params(s, **params)
    return CisdEnergies.apply(*(tensors[k] for k in KEYS), s, sysc, par, symR, nroot)


KEYS3 = ("ijkl", "ijka", "abij", "iabj", "abci", "abcd", "eorb")


class Cpsd3Energies(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ijkl, ijka, abij, iabj, abci, abcd, eorb, s, sysc, par, symR, nroot):
        t = dict(zip(KEYS3, (ijkl, ijka, abij, iabj, abci, abcd, eorb)))
        w0, w2, w3, L = api.cpsd3_energies(s, sysc, api.integrals_struct(t), par, symR, nroot)
        ctx.save_for_backward(ijkl, ijka, abij, iabj, abci, abcd, eorb, L)
        ctx.meta = (sysc, par, symR, w0)
        return torch.from_numpy(w0), torch.from_numpy(w2), torch.from_numpy(w3)

    @staticmethod
    def backward(ctx, g0, g2, g3):
        *lists, L = ctx.saved_tensors
        sysc, par, symR, w0 = ctx.meta
        n = len(w0)
        g = [np.zeros(n) if x is None else x.detach().cpu().double().numpy() for x in (g0, g2, g3)]
        t = dict(zip(KEYS3, lists))
        grads = {k: torch.zeros_like(v) for k, v in t.items()}
        api.cpsd3_gradient(sysc, api.integrals_struct(t), par, symR, w0, L, *g, grads)
        return tuple(grads[k] for k in KEYS3) + (None,) * 5


def cpsd3_energies(s, tensors, symR, nroot, **params):
    """(w0, w2, w3) of nroot roots of irrep symR; tensors: dict of float64
    CUDA tensors with keys ijkl, ijka, abij, iabj, abci, abcd, eorb."""
    sysc = api.make_system(s)
    par = api.make_params(s, **params)
    return Cpsd3Energies.apply(*(tensors[k] for k in KEYS3), s, sysc, par, symR, nroot)
