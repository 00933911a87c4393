"""CPU oracle of BuildSC -- TEST INFRASTRUCTURE ONLY (the checker of phf_pcc_b200's BuildSC path).

Restates in numpy the reference's grid-projected "S x C" product of the projected coupled-cluster
linear-dependency solver (LinDep.py:71-76):

* ``buildsc``      -- BuildSC, PHF_fort/PHFTools.f90:464-537: the grid loop il, iy, ipg;
                      R = R1 R2 Rpg, RDM of the reference determinant (newMO = [I; 0]);
                      c1 and c2 transformed with R^H (ao2mo2 :390-398, ao2mo4 :400-462);
                      BuildSC_Vec; weights weightsp s_w sum_{m,n,p,q} weightpg conj(fsp_m) fsp_n
                      conj(fpg_p) fpg_q (the Wigner factor is computed and then set to one at
                      :517-518, which this restatement keeps); every sum divided by the
                      projected overlap
* ``buildsc_vec``  -- BuildSC_Vec, PHF_fort/BuildSC_dr.f90:8-1244: the contraction sequence of
                      the vector (c0, c1, c2) with the transition density Y, in its order

Indices follow the Fortran arrays: a numpy array A[a, b, c, d] is A(a, b, c, d).  The reference's
BuildSC exists only as Fortran behind a closed f2py binary, so no reference output pins this
restatement; it is checked for the algebraic properties its tests state (linearity in the vector,
the c0 channel alone, the identity rotation) and transcribes the loops one statement per line.
"""
from __future__ import annotations

import numpy as np

from .phf_oracle import mo_transform_2, rdm


def buildsc_vec(c0, c1, c2, Y):
    """BuildSC_Vec (PHF_fort/BuildSC_dr.f90:8-1244): (t0, t1, t2) from (c0, c1, c2) and Y."""
    e = np.einsum
    tau0 = c2 - e("bacd->abcd", c2)
    tau1 = e("cd,dabc->ab", Y, tau0)
    tau2 = -tau1
    tau6 = -tau1
    tau8 = -e("ab,ba->", Y, tau1)
    t2 = tau8 * e("ac,bd->abcd", Y, Y)
    t2 -= tau8 * e("ad,bc->abcd", Y, Y)
    tau13 = -tau1
    tau5 = e("cd,adcb->ab", Y, tau0)
    tau6 -= tau5
    tau13 -= tau5
    tau14 = e("ac,cb->ab", Y, tau13)
    tau15 = e("ca,bc->ab", Y, tau14)
    tau16 = -e("ac,db->abcd", Y, tau15)
    tau21 = e("ca,bc->ab", Y, tau13)
    tau22 = e("ab,cd->abcd", Y, tau21)
    tau2 += c1
    tau3 = e("ab,ba->", Y, tau2)
    t0 = tau3
    t1 = tau3 * Y
    tau4 = -c2 + e("bacd->abcd", c2)
    tau7 = -e("cd,dabc->ab", Y, tau4)
    tau7 -= e("cd,adcb->ab", Y, tau4)
    tau6 += c1
    tau7 += e("ac,cb->ab", Y, tau6)
    tau7 -= c1
    t1 = t1 - e("cb,ac->ab", Y, tau7)
    tau9 = e("ea,bcde->abcd", Y, c2)
    tau10 = e("ea,bcde->abcd", Y, tau9)
    tau11 = e("ae,bcde->abcd", Y, tau10)
    tau12 = e("ae,bcde->abcd", Y, tau11)
    tau16 += tau12
    t2 += tau16
    t2 -= e("abdc->abcd", tau16)
    t2 -= e("bacd->abcd", tau16)
    t2 += e("badc->abcd", tau16)
    tau19 = -tau10 + e("abdc->abcd", tau10)
    tau20 = e("ae,bcde->abcd", Y, tau19)
    tau22 -= tau20
    t2 += e("acdb->abcd", tau22)
    t2 -= e("adcb->abcd", tau22)
    t2 -= e("bcda->abcd", tau22)
    t2 += e("bdca->abcd", tau22)
    t2 += e("cdab->abcd", tau10)
    t2 -= e("cdba->abcd", tau10)
    t2 -= e("dcab->abcd", tau10)
    t2 += e("dcba->abcd", tau10)
    tau17 = e("ca,bc->ab", Y, c1)
    tau18 = e("ac,bc->ab", Y, tau17)
    t2 -= e("ac,bd->abcd", Y, tau18)
    t2 += e("bc,ad->abcd", Y, tau18)
    t2 += e("ac,db->abcd", Y, tau17)
    t2 -= e("bc,da->abcd", Y, tau17)
    tau23 = e("ba,ab->", Y, c1)
    tau27 = tau23 * Y.T
    tau24 = e("ac,cb->ab", Y, c1)
    tau25 = tau24 - c1
    tau26 = e("ca,bc->ab", Y, tau25)
    tau27 = tau27 - tau26
    tau27 = tau27 + c0 * Y.T
    t2 += e("bd,ca->abcd", Y, tau27)
    t2 -= e("ad,cb->abcd", Y, tau27)
    t0 = t0 + c0
    t1 = t1 + c0 * Y
    return complex(t0), t1, t2


def buildsc(c0, c1, c2, nocc, ngrid, qj, r1, r2, rpg, roota, rootb, rooty, weightsp, weightpg, fsp, fpg,
            point_list=None):
    """BuildSC (PHF_fort/PHFTools.f90:464-537).  Returns (t0, t1 (M, M), t2 (M, M, M, M)) divided by
    the projected overlap.  ``point_list``: flattened grid points ((il ny + iy) npg + ipg) to sum over
    (all by default; the overlap then covers the same points)."""
    M = c1.shape[0]
    nl, ny = int(ngrid[0]), int(ngrid[1])
    npg = rpg.shape[0]
    fsp = np.atleast_1d(np.asarray(fsp, dtype=np.complex128))
    fpg = np.atleast_1d(np.asarray(fpg, dtype=np.complex128))
    newMO = np.zeros((M, nocc), dtype=np.complex128)
    newMO[:nocc, :nocc] = np.eye(nocc)
    # sum_{m,n} conj(fsp_m) fsp_n (one term per Wigner pair, the factor itself set to one)
    fsum = np.conj(fsp).sum() * fsp.sum()
    del qj, roota, rootb, rooty  # the Wigner factor's arguments: computed and discarded (:516-518)
    t0, t1, t2 = 0j, np.zeros((M, M), complex), np.zeros((M, M, M, M), complex)
    ovlp = 0j
    pts = range(nl * ny * npg) if point_list is None else point_list
    for w in pts:
        il, iy, ipg = w // (ny * npg), (w // npg) % ny, w % npg
        R = r1[il] @ r2[iy] @ rpg[ipg]
        rho, s = rdm(R, newMO)
        U = R.conj().T
        c1t = U.conj().T @ c1 @ U                       # ao2mo2(c1, R^H)
        c2t = mo_transform_2(c2, U)                     # ao2mo4(c2, R^H)
        a0, a1, a2 = buildsc_vec(c0, c1t, c2t, rho)
        s = weightsp[il, iy] * s
        wpg = sum(weightpg[ipg, p, q] * np.conj(fpg[p]) * fpg[q] for p in range(len(fpg)) for q in range(len(fpg)))
        w_ = wpg * fsum
        t0 += a0 * s * w_
        t1 += a1 * s * w_
        t2 += a2 * s * w_
        ovlp += s * w_
    return t0 / ovlp, t1 / ovlp, t2 / ovlp
