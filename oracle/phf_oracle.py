"""CPU oracle for the projected-HF grid kernel -- TEST INFRASTRUCTURE ONLY.

This module is the checker.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it; the product (``phf_pcc_b200``) never
does, and it is never the thing measured as the GPU result.

It restates, in numpy, the reference's FP64 algorithm for ``phftools.buildhsg`` and
``phftools.localg``:

* ``buildhsg``  -- PHF_fort/PHFTools.f90:10-201 (BuildHSG), loop order il, iy, ipg,
                   accumulation of weighted h, s, g, rho*s into (nci, nci[, M, M]) slots,
                   CmplxConj == 2 four-density branch (:95-119, :153-163, :174-179)
* ``rdm``       -- PHFTools.f90:249-263 (RDM); ``rdm_conj`` -- :265-279 (RDMConj)
* ``make_gamma``-- PHFTools.f90:310-337 (MakeGamma), dense <ij||kl> contraction;
                   ``make_gamma_chol`` is the identical J - K form from Cholesky vectors
* ``makeh``     -- PHFTools.f90:339-348; ``kernels`` -- :281-289; ``gradient`` -- :291-308
* ``localg``    -- PHFTools.f90:203-247
* ``eigen_solver`` / ``vec_decomp`` -- PHFTools.py:8-26
* ``hermiticity_violation`` -- the check of PHFTools.f90:195-200

Parity of this restatement is pinned by ``tests/golden`` fixtures that were produced by
the reference's own Python functions (PHFTools.py Rdm/Kernels/Gradient/LocalG/
EigenSolver/VecDecomp, SpinSymm.py, WignerMat.py).  The reference's LAPACK
(ZGETRF/ZGETRI in a closed library) is stood in for by numpy.linalg.inv/det.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "rdm", "rdm_conj", "make_gamma", "make_gamma_chol", "makeh", "kernels", "gradient",
    "wigner_D", "buildhsg", "localg", "eigen_solver", "vec_decomp", "hermiticity_violation",
    "dense_htwo_from_chol", "mo_transform_1", "mo_transform_2", "energy_and_gradient",
]


def rdm(R, MO):
    """RDM (PHFTools.f90:249-263): tmp = R MO, M = MO^H tmp, rho = tmp M^-1 MO^H, det M."""
    tmp = R @ MO
    Mm = MO.conj().T @ tmp
    Minv = np.linalg.inv(Mm)
    det = np.linalg.det(Mm)
    rho = (tmp @ Minv) @ MO.conj().T
    return rho, det


def rdm_conj(R, MO):
    """RDMConj (PHFTools.f90:265-279): as rdm with R conj(MO) as the ket."""
    tmp = R @ MO.conj()
    Mm = MO.conj().T @ tmp
    Minv = np.linalg.inv(Mm)
    det = np.linalg.det(Mm)
    rho = (tmp @ Minv) @ MO.conj().T
    return rho, det


def make_gamma(H2, rho):
    """MakeGamma (PHFTools.f90:310-337): gamma_ik = sum_jl H2_ijkl rho_lj."""
    return np.einsum("ijkl,lj->ik", H2, rho, optimize=True)


def make_gamma_chol(Bso, rho):
    """Gamma = J - K from spin-orbital Cholesky vectors Bso (L, M, M) with
    (ik|jl) = sum_L Bso[L,i,k] Bso[L,j,l]; identical to make_gamma with
    H2 = <ij||kl> = (ik|jl) - (il|jk)."""
    d = np.einsum("Ljl,lj->L", Bso, rho, optimize=True)
    J = np.einsum("L,Lik->ik", d, Bso, optimize=True)
    K = np.einsum("Lil,lj,Ljk->ik", Bso, rho, Bso, optimize=True)
    return J - K


def makeh(H1, gama, rho):
    """Makeh (PHFTools.f90:339-348): h = sum(H1^T * rho) + sum(gama * rho^T)/2."""
    return np.sum(H1.T * rho) + np.sum(gama * rho.T) / 2.0


def kernels(H1, gama, rho, det):
    """Kernels (PHFTools.f90:281-289): det * Makeh."""
    return makeh(H1, gama, rho) * det


def gradient(H1, gama, rho, det):
    """Gradient (PHFTools.f90:291-308): det * [(I - rho)(H1 + gama) rho + h rho]."""
    M = rho.shape[0]
    h = makeh(H1, gama, rho)
    G = (H1 + gama) @ rho
    G = (np.eye(M) - rho) @ G
    G = G + h * rho
    return G * det


def wigner_D(j, n, m, alpha, beta, gamma):
    """Wignerfac (PHFTools.f90:350-376)."""
    pre = math.sqrt(math.factorial(j + n) * math.factorial(j - n) * math.factorial(j + m) * math.factorial(j - m))
    acc = 0.0
    for s in range(max(0, m - n), min(j + m, j - n) + 1):
        p1, p2, p3 = n - m + s, 2 * j + m - n - 2 * s, n - m + 2 * s
        num = (-1.0) ** p1 * math.cos(beta / 2) ** p2 * math.sin(beta / 2) ** p3
        den = math.factorial(j + m - s) * math.factorial(s) * math.factorial(n - m + s) * math.factorial(j - n - s)
        acc += num / den
    return complex(np.exp(-1j * n * alpha) * pre * acc * np.exp(-1j * m * gamma))


def mo_transform_1(A, U):
    """ao2mo(., U, 2) of ao2mo.py:4-10: U^H A U."""
    return U.conj().T @ A @ U


def mo_transform_2(H2, U):
    """ao2mo(., U, 4) of ao2mo.py:4-10: sum U*_ai U*_bj H_abcd U_ck U_dl."""
    Uc = U.conj()
    t = np.einsum("abcd,ai->ibcd", H2, Uc, optimize=True)
    t = np.einsum("ibcd,bj->ijcd", t, Uc, optimize=True)
    t = np.einsum("ijcd,ck->ijkd", t, U, optimize=True)
    return np.einsum("ijkd,dl->ijkl", t, U, optimize=True)


def dense_htwo_from_chol(B):
    """Spin-orbital antisymmetrised <ij||kl> from spatial Cholesky vectors B (L, n, n).

    (pq|rs) = sum_L B[L,p,q] B[L,r,s]; spin blocks as Main_PHF.py:22-29, then
    Mulliken -> Dirac with antisymmetrisation as makeH.py:63-67."""
    L, n, _ = B.shape
    M = 2 * n
    eri = np.einsum("Lpq,Lrs->pqrs", B, B, optimize=True)
    Hm = np.zeros((M, M, M, M))
    a, b = slice(0, n), slice(n, M)
    Hm[a, a, a, a] = eri
    Hm[b, b, b, b] = eri
    Hm[b, b, a, a] = eri
    Hm[a, a, b, b] = eri
    tmp = np.einsum("ijkl->ikjl", Hm)
    return tmp - np.einsum("ijkl->ijlk", tmp)


def chol_spin_orbital(B, U=None):
    """Spin-orbital Cholesky vectors I2 (x) B_L, optionally transformed to a basis U: U^H B U."""
    L, n, _ = B.shape
    M = 2 * n
    Bso = np.zeros((L, M, M), dtype=np.complex128 if U is not None else np.float64)
    Bso[:, :n, :n] = B
    Bso[:, n:, n:] = B
    if U is not None:
        Bso = np.einsum("ai,Lab,bk->Lik", U.conj(), Bso, U, optimize=True)
    return Bso


def buildhsg(HOne, HTwo, Ref, Z, ngrid, nci, CmplxConj, ncisp, NOcc, R1, R2, Rpg, weightsp, weightpg,
             roota, rootb, rooty, QJ, SP, npg, ncipg, NSO, Bso=None, omega_subset=None):
    """BuildHSG (PHFTools.f90:10-201) without the Hermiticity STOP.

    Gamma comes from the dense HTwo (MakeGamma) or, when ``Bso`` is given, from
    spin-orbital Cholesky vectors in the same (MO) basis.  ``omega_subset`` restricts
    the sum to a list of (il, iy, ipg) points (used for bounded CPU timing samples).
    Returns (Hmat, Smat, Gradmat, Rdmmat) with shapes (nci, nci), (nci, nci),
    (nci, nci, M, M), (nci, nci, M, M)."""
    M = NSO
    Zt = np.array(Z, dtype=np.complex128)
    if CmplxConj == 0:
        Zt = Zt.real.astype(np.complex128)
    newMO = np.zeros((M, NOcc), dtype=np.complex128)
    newMO[:NOcc, :NOcc] = np.eye(NOcc)
    newMO[NOcc:, :] = Zt
    Hmat = np.zeros((nci, nci), dtype=np.complex128)
    Smat = np.zeros((nci, nci), dtype=np.complex128)
    Gradmat = np.zeros((nci, nci, M, M), dtype=np.complex128)
    Rdmmat = np.zeros((nci, nci, M, M), dtype=np.complex128)
    d = ncisp * ncipg

    def gam(rho):
        return make_gamma(HTwo, rho) if Bso is None else make_gamma_chol(Bso, rho)

    points = omega_subset
    if points is None:
        points = [(il, iy, ipg) for il in range(ngrid[0]) for iy in range(ngrid[1]) for ipg in range(npg)]
    for (il, iy, ipg) in points:
        Rtmp = R1[il] @ R2[iy] @ Rpg[ipg]
        R = Ref.conj().T @ Rtmp @ Ref
        rho0, s0 = rdm(R, newMO)
        g0m = gam(rho0)
        h0 = kernels(HOne, g0m, rho0, s0)
        g0 = gradient(HOne, g0m, rho0, s0)
        if CmplxConj == 2:
            rho1, s1 = rdm_conj(R, newMO)
            g1m = gam(rho1)
            h1 = kernels(HOne, g1m, rho1, s1)
            g1 = gradient(HOne, g1m, rho1, s1)
            rho0c, s0c = rdm(R, newMO.conj())
            g0c = gradient(HOne, gam(rho0c), rho0c, s0c)
            rho1c, s1c = rdm_conj(R, newMO.conj())
            g1c = gradient(HOne, gam(rho1c), rho1c, s1c)
        else:
            h1, g1, s1, rho1 = h0, g0, s0, rho0
            g0c, s0c, rho0c = g0, s0, rho0
            g1c, s1c, rho1c = g0, s0, rho0
        wsp = weightsp[il, iy]
        rho0 = rho0 * wsp * s0
        rho1 = rho1 * wsp * s1
        rho0c = rho0c * wsp * s0c
        rho1c = rho1c * wsp * s1c
        h0 = wsp * h0
        h1 = wsp * h1
        s0 = wsp * s0
        s1 = wsp * s1
        g0 = g0 * wsp
        g1 = g1 * wsp
        g0c = g0c * wsp
        g1c = g1c * wsp
        for ni in range(-QJ, QJ + 1):
            for nj in range(-QJ, QJ + 1):
                if SP == 2:
                    wig = wigner_D(QJ, ni, nj, roota[il], rootb[iy], rooty[il])
                else:
                    wig = wigner_D(QJ, ni, nj, roota[il], rootb[il], rooty[iy])
                for p in range(ncipg):
                    for q in range(ncipg):
                        w = weightpg[ipg, p, q] * wig
                        m = ni + QJ + p * ncisp
                        n = nj + QJ + q * ncisp
                        Hmat[m, n] += h0 * w
                        Smat[m, n] += s0 * w
                        Gradmat[m, n] += g0 * w
                        Rdmmat[m, n] += rho0 * w
                        if CmplxConj == 2:
                            Hmat[m, n + d] += h1 * w
                            Smat[m, n + d] += s1 * w
                            Gradmat[m, n + d] += g1 * w
                            Rdmmat[m, n + d] += rho1 * w
                            Gradmat[m + d, n] += g1c * w
                            Rdmmat[m + d, n] += rho1c * w
                            Gradmat[m + d, n + d] += g0c * w
                            Rdmmat[m + d, n + d] += rho0c * w
    if CmplxConj == 2:
        Hmat[d:, :d] = Hmat[:d, d:].conj().T
        Smat[d:, :d] = Smat[:d, d:].conj().T
        Hmat[d:, d:] = Hmat[:d, :d]
        Smat[d:, d:] = Smat[:d, :d]
    return Hmat, Smat, Gradmat, Rdmmat


def hermiticity_violation(Hmat, Smat, tol=1e-5):
    """True when the reference would STOP "Not Hermitian" (PHFTools.f90:195-200)."""
    w1 = np.max(np.abs(np.imag(Hmat.conj().T - Hmat)))
    w2 = np.max(np.abs(np.imag(Smat.conj().T - Smat)))
    return bool(w1 > np.max(np.abs(Hmat)) * tol or w2 > np.max(np.abs(Smat)) * tol)


def localg(Gradmat, Rdmmat, Smat, E0, fsp, fpg, fk, CmplxConj, NSO, nci, ncisp, ncipg):
    """LocalG (PHFTools.f90:203-247): G = (sum f*f Grad - E0 sum f*f Rdm) / sum f*f S (full M x M)."""
    M = NSO
    G = np.zeros((M, M), dtype=np.complex128)
    Rdm = np.zeros((M, M), dtype=np.complex128)
    Ovlp = 0.0 + 0.0j
    fk = np.atleast_1d(fk)
    for ni in range(ncisp):
        for nj in range(ncisp):
            for p in range(ncipg):
                for q in range(ncipg):
                    m = ni + p * ncisp
                    n = nj + q * ncisp
                    f = np.conj(fsp[ni]) * fsp[nj] * np.conj(fpg[p]) * fpg[q]
                    G += f * np.conj(fk[0]) * fk[0] * Gradmat[m, n]
                    Rdm += f * np.conj(fk[0]) * fk[0] * Rdmmat[m, n]
                    Ovlp += f * np.conj(fk[0]) * fk[0] * Smat[m, n]
                    if CmplxConj == 2:
                        d = ncisp * ncipg
                        G += f * np.conj(fk[1]) * fk[1] * np.conj(Gradmat[m + d, n + d])
                        Rdm += f * np.conj(fk[1]) * fk[1] * np.conj(Rdmmat[m + d, n + d])
                        Ovlp += f * np.conj(fk[1]) * fk[1] * Smat[m + d, n + d]
                        G += f * np.conj(fk[0]) * fk[1] * Gradmat[m, n + d]
                        Rdm += f * np.conj(fk[0]) * fk[1] * Rdmmat[m, n + d]
                        Ovlp += f * np.conj(fk[0]) * fk[1] * Smat[m, n + d]
                        G += f * np.conj(fk[0]) * fk[1] * np.conj(Gradmat[m + d, n])
                        Rdm += f * np.conj(fk[0]) * fk[1] * np.conj(Rdmmat[m + d, n])
                        Ovlp += f * np.conj(fk[1]) * fk[0] * Smat[m + d, n]
    return (G - E0 * Rdm) / Ovlp


def eigen_solver(H, S, tol=1e-6):
    """EigenSolver (PHFTools.py:8-18): canonical orthogonalisation then eigh."""
    evals, evecs = np.linalg.eigh(S)
    Dim = len(evals)
    invS = [1 / np.sqrt(abs(i)) for i in evals if (np.abs(i) > tol)]
    dim = len(invS)
    X = evecs[:, Dim - dim:] @ np.diag(invS)
    h = X.conj().T @ H @ X
    e, v = np.linalg.eigh(h)
    return e, X @ v


def vec_decomp(vec, ncisp, ncipg, ncik):
    """VecDecomp (PHFTools.py:20-26)."""
    Mv = vec.reshape((ncisp * ncipg, ncik), order="F")
    fk = Mv[0, :] / Mv[0, 0]
    Mv = Mv[:, 0].reshape((ncisp, ncipg), order="F")
    fpg = Mv[0, :] / Mv[0, 0]
    fsp = Mv[:, 0]
    return fsp, fpg, fk


def energy_and_gradient(HOne, HTwo, Ref, Z, grid_args, Bso=None):
    """EandG's kernel part (PHF.py:70-78): buildhsg -> EigenSolver -> VecDecomp -> localg.

    ``grid_args`` is a dict with the buildhsg keyword arguments other than HOne, HTwo,
    Ref, Z.  Returns (E0, G_full (M x M), Hmat, Smat)."""
    a = grid_args
    Hm, Sm, Gm, Rm = buildhsg(HOne, HTwo, Ref, Z, Bso=Bso, **a)
    ncik = 2 if a["CmplxConj"] == 2 else 1
    e, v = eigen_solver(Hm, Sm)
    fsp, fpg, fk = vec_decomp(v[:, 0], a["ncisp"], a["ncipg"], ncik)
    G = localg(Gm, Rm, Sm, e[0], fsp, fpg, fk, a["CmplxConj"], a["NSO"], a["nci"], a["ncisp"], a["ncipg"])
    return e[0], G, Hm, Sm
