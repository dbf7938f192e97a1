"""torch.autograd binding of the energy adjoint (checks only).

The ground-state energy of the selected-CI problem is a function of the
integral entries as an FCIDUMP lists them: one value per unordered one-electron
pair (p >= q, setting h_pq and h_qp) and one per 8-fold two-electron class. By
Hellmann-Feynman its gradient is the contraction pattern of the 1-/2-RDM of the
converged vector; sbdx_energy_backward computes it on the GPU (recomputing the
connectivity and the RDMs from the vector). This Function exposes that pair as
forward (a Davidson solve through the C-ABI) and backward (the adjoint kernel).
"""
from __future__ import annotations

import numpy as np
import torch

from . import SBDX_FP64, Context


def tril_pack(h: np.ndarray) -> np.ndarray:
    L = h.shape[0]
    p, q = np.tril_indices(L)
    return h[p, q].copy()


def tril_unpack(v: np.ndarray, L: int) -> np.ndarray:
    h = np.zeros((L, L))
    p, q = np.tril_indices(L)
    h[p, q] = v
    h[q, p] = v
    return h


class SelectedCIEnergy(torch.autograd.Function):
    """E(h_tri, eri) for a fixed alpha x beta basis held by `context`."""

    @staticmethod
    def forward(fctx, h_tri, eri, context: Context, L: int, I0: float, solve: dict):
        h = tril_unpack(h_tri.detach().cpu().double().numpy(), L)
        context.set_integrals(L, I0, h, eri.detach().cpu().double().numpy())
        info, W = context.davidson(**solve)
        if not info.converged:
            raise RuntimeError(f"Davidson did not converge (residual {info.residual:.3e})")
        fctx.context, fctx.W, fctx.L = context, W, L
        return torch.tensor(info.energy, dtype=torch.float64)

    @staticmethod
    def backward(fctx, gE):
        dh, deri = fctx.context.energy_backward(fctx.W)
        g_h = torch.from_numpy(tril_pack(dh.reshape(fctx.L, fctx.L))) * gE
        g_eri = torch.from_numpy(deri) * gE
        return g_h, g_eri, None, None, None, None


def energy(context: Context, h_tri: torch.Tensor, eri: torch.Tensor, L: int, I0: float, **solve):
    solve = {"max_it": 50, "max_nb": 12, "eps": 1e-10, "precision": SBDX_FP64, **solve}
    return SelectedCIEnergy.apply(h_tri, eri, context, L, I0, solve)
