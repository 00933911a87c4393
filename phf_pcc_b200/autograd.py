"""Projected energy as a differentiable function of the determinant C (torch.autograd).

E(C) is the projected energy of PHF.py's EandG (PHF.py:70-77): the lowest root of
Hmat c = E Smat c (EigenSolver, PHFTools.py:8-18), which for one projection channel
(nci = 1) is E = Re H / |Re S|.  Its derivative is the reference's gradient (LocalG,
PHF_fort/PHFTools.f90:203-247) written for C itself instead of the Thouless Z:

    dE/dC* = (sum f* f Yg - E sum f* f Yr) / sum f* f S

with Yg, Yr the weighted grid sums that the CUDA pipeline accumulates in the same pass as
H and S (the adjoint of rho_w = R_w C (C^H R_w C)^-1 C^H contracted with the per-point
Fock matrix).  Nothing per grid point is stored between forward and backward: the saved
state is two M x N matrices.  ``mode="recompute"`` keeps only C from the forward and
re-runs the pass in backward (for callers that evaluate many energies and few gradients).

The reference's gradient is the derivative through C^H (the bra) only; it equals dE/dC*
when the grid sum is exactly Hermitian.  A plan created with gradient="exact" also accumulates
the derivative through R C (the ket) and returns the exact dE/dC* for any grid; that is the
gradient finite differences see.

PyTorch's gradient of a real function of complex C is 2 dE/dC* (conjugate Wirtinger
convention), which is what ``backward`` returns.
"""
from __future__ import annotations

import numpy as np
import torch

from .api import Plan

__all__ = ["ProjectedEnergy", "projected_energy", "energy_and_gradient"]


def _combine(hs, yg, yr, nci, ncisp, ncipg, tol=1e-6, exact=False):
    """Energy and dE/dC* from the slot accumulators (EigenSolver + VecDecomp + LocalG).

    With ``exact`` the accumulators are the symmetrised bra+ket sums of a plan created with
    gradient="exact" and the result is the exact derivative of E = Re H / |Re S|."""
    if nci == 1:
        H, S = hs[0, 0], hs[0, 1]
        s = S.real.abs()
        E = H.real / s
        if exact:
            G = (yg[0] - E * torch.sign(S.real) * yr[0]) / s
        else:
            G = (yg[0] - E * yr[0]) / S
        return E, G
    # several channels: the small generalized eigenproblem on the host (nci x nci)
    Hm = hs[:, 0].reshape(nci, nci).T.cpu().numpy()   # slot a = m + nci n
    Sm = hs[:, 1].reshape(nci, nci).T.cpu().numpy()
    w, V = np.linalg.eigh(Sm)
    keep = np.abs(w) > tol
    X = V[:, keep] / np.sqrt(np.abs(w[keep]))[None, :]
    e, U = np.linalg.eigh(X.conj().T @ Hm @ X)
    vec = X @ U[:, 0]
    Mv = vec.reshape((ncisp * ncipg, 1), order="F")
    Mv = Mv[:, 0].reshape((ncisp, ncipg), order="F")
    fpg = Mv[0, :] / Mv[0, 0]
    fsp = Mv[:, 0]
    coef = np.zeros((nci, nci), dtype=np.complex128)
    for ni in range(ncisp):
        for nj in range(ncisp):
            for p in range(ncipg):
                for q in range(ncipg):
                    coef[ni + p * ncisp, nj + q * ncisp] += np.conj(fsp[ni]) * fsp[nj] * np.conj(fpg[p]) * fpg[q]
    c = torch.from_numpy(coef.T.reshape(-1)).to(yg.device)  # slot order a = m + nci n
    ovlp = (c * hs[:, 1]).sum()
    E = torch.tensor(float(e[0]), dtype=torch.float64, device=yg.device)
    G = ((c[:, None, None] * yg).sum(0) - E * (c[:, None, None] * yr).sum(0)) / ovlp
    return E, G


class ProjectedEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, C, plan, mode="fused"):
        hs, yg, yr = plan.eval_device(C.detach())
        E, G = _combine(hs, yg, yr, plan.nci, plan._g.ncisp, plan._g.ncipg, exact=plan.gradient == "exact")
        ctx.plan = plan
        ctx.mode = mode
        if mode == "fused":
            ctx.save_for_backward(G)
        else:
            ctx.save_for_backward(C.detach())
        return E

    @staticmethod
    def backward(ctx, gE):
        (saved,) = ctx.saved_tensors
        if ctx.mode == "fused":
            G = saved
        else:
            hs, yg, yr = ctx.plan.eval_device(saved)
            _, G = _combine(hs, yg, yr, ctx.plan.nci, ctx.plan._g.ncisp, ctx.plan._g.ncipg,
                            exact=ctx.plan.gradient == "exact")
        return 2.0 * gE * G, None, None


def projected_energy(C: torch.Tensor, plan: Plan, mode: str = "fused") -> torch.Tensor:
    """Projected energy E(C) (differentiable in C, a complex128 CUDA tensor (M, N))."""
    return ProjectedEnergy.apply(C, plan, mode)


def energy_and_gradient(C: torch.Tensor, plan: Plan):
    """(E, dE/dC*) for a device-resident C, one pass of the pipeline."""
    hs, yg, yr = plan.eval_device(C)
    return _combine(hs, yg, yr, plan.nci, plan._g.ncisp, plan._g.ncipg, exact=plan.gradient == "exact")
