"""CPU oracle for the projected coupled-cluster grid kernel -- TEST INFRASTRUCTURE ONLY.

This module is the checker for ``phf_pbarhbarolap``.  Only ``tests/`` and the CPU-baseline
leg of ``bench.py`` may import it; the product (``phf_pcc_b200``) never does.

It restates, in numpy, the reference's FP64 grid kernel of projected CCSD
(SUCCSD_Boson_cmplx/, Fortran compiled into the PUCC_X2 extension):

* ``pbarhbarolap``  -- FPUCC.f90:14-272 (PbarHbarOlap): loop il, iy, ipg (and the Rk(2) pass
                       for ncik = 2, :186-228), per-point weight = sum over the Wigner pairs
                       (m, n) and point-group components (p, q) (:160-176), ProjSz of the sums
                       for SP = 2 (:231-234)
* ``eval_kernel``   -- FPUCC.f90:529-602 (EvalKernel)
* ``dstt2``         -- FPUCC_Tools.f90:697-722 (DSTT2) = ``proj_t1`` (:676-695) +
                       ``build_w`` (PCCCI.f90:14-40) = ``trans_t2`` (PCCCI.f90:100-276) + ``ci2cc``
                       (PCCCI.f90:72-98)
* ``build_thouless_z`` -- FPUCC_Tools.f90:50-93; ``int_tran4_sim`` -- IntTrans.f90:486-572
* ``mkfock_mo``     -- UHF.f90:461-500
* ``build_kern_sd`` -- FPUCC_Tools.f90:291-436 (BuildKernSD)
* ``cc_energy``     -- CCRes.f90:9-29; ``cc_itms`` -- CCRes.f90:355-537; ``cc_res12`` --
                       CCRes.f90:164-353; ``asymm2`` -- CCRes.f90:31-70; ``aperm`` -- :120-162
* ``ccsd_t_energy`` -- CCSD_T.f90:10-108 (CCSD_T_Ene, get_wv, Perm3, DirectSum3)
* ``proj_sz1`` / ``proj_sz2_vo`` -- FPUCC_Tools.f90:150-234
* ``wigner``        -- Wrappers.f90:769-797 (argument order J, N, M as declared there)

Every array is indexed like the Fortran one, with the occupied range first: a vo array
T1[a, i] is T1(NOcc+1+a, 1+i), a vvoo array T2[a, b, i, j] is T2(NOcc+1+a, NOcc+1+b, 1+i, 1+j),
and NSO-sized arrays use the full range.  InvertC / determinantC (LAPACK in a closed library) are
stood in for by numpy.linalg.inv / det.

Parity unpinned: the reference's PCC kernel exists only as Fortran behind a closed binary and has
no Python twin, so no reference output pins it.  The restatement follows the Fortran statement by
statement (each At_dot_B / A_dot_Bt / Transpose2 written out as the index contraction it performs,
including the reuse of a name for a transposed copy, e.g. ``oovv`` in TransT2 after :167), and the
tests check it against independent facts: the CCSD residual and energy against a determinant-space
evaluation of <Phi_ij..^ab..| exp(-T) H exp(T) |Phi_0> (tests/test_pcc_oracle.py), the
Thouless factor against det, and the identity rotation.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "wigner", "build_thouless_z", "proj_t1", "int_tran4_sim", "mkfock_mo", "trans_t2", "ci2cc", "build_w", "dstt2",
    "asymm2", "aperm", "cc_energy", "cc_itms", "cc_res12", "ccsd_t_energy", "build_kern_sd", "proj_sz1", "proj_sz2_vo",
    "eval_kernel", "point_weights", "pbarhbarolap", "pbarhbar_res_from_olap", "make_pcc_problem",
]

ES = dict(optimize=True)


def wigner(J, N, M, alpha, beta, gama):
    """Wigner (Wrappers.f90:769-797): exp(-i N alpha) d^J_{NM}(beta) exp(-i M gama)."""
    n, m, j = N, M, J
    fac = math.sqrt(math.gamma(j + n + 1) * math.gamma(j - n + 1) * math.gamma(j + m + 1) * math.gamma(j - m + 1))
    d = 0.0
    for s in range(max(0, m - n), min(j + m, j - n) + 1):
        p1, p2, p3 = n - m + s, 2 * j + m - n - 2 * s, n - m + 2 * s
        numer = (-1.0) ** p1 * math.cos(beta / 2) ** p2 * math.sin(beta / 2) ** p3
        denom = math.gamma(j + m - s + 1) * math.gamma(s + 1) * math.gamma(n - m + s + 1) * math.gamma(j - n - s + 1)
        d += numer / denom
    return complex(np.exp(-1j * n * alpha) * d * fac * np.exp(-1j * m * gama))


def build_thouless_z(MO1, MO2, o):
    """BuildThoulessZ (FPUCC_Tools.f90:50-93): Tran = MO1^H MO2, L = Tran[:o, :o],
    Y = Tran[o:, :o]; Z = Y L^-1, Olap = det L."""
    Tran = MO1.conj().T @ MO2
    L, Y = Tran[:o, :o], Tran[o:, :o]
    return np.linalg.det(L), Y @ np.linalg.inv(L)


def proj_t1(R, T1, o):
    """ProjT1 (FPUCC_Tools.f90:676-695): MO2 = R [1 0; T1 1] and its Thouless form against 1."""
    M = R.shape[0]
    MO2 = np.eye(M, dtype=complex)
    MO2[o:, :o] = T1
    return build_thouless_z(np.eye(M, dtype=complex), R @ MO2, o)


def int_tran4_sim(ERI, RMat):
    """IntTran4Sim (IntTrans.f90:486-572): index 4, then 3 with R^-1 (ket side), index 2, then 1
    with R (bra side): E'(p,q,r,s) = sum R(p,a) R(q,b) E(a,b,c,d) R^-1(c,r) R^-1(d,s)."""
    InvR = np.linalg.inv(RMat)
    E2 = np.einsum("abcd,ds->abcs", ERI, InvR, **ES)
    E = np.einsum("abcs,cr->abrs", E2, InvR, **ES)
    E2 = np.einsum("abrs,qb->aqrs", E, RMat, **ES)
    return np.einsum("pa,aqrs->pqrs", RMat, E2, **ES)


def mkfock_mo(OneH, ERI, o):
    """MKFock_MO (UHF.f90:461-500): F = h + sum_i <p i|q i>, E = sum_i h_ii + sum_ij <ij|ij>/2."""
    F = OneH + np.einsum("piqi->pq", ERI[:, :o, :, :o])
    E = np.trace(OneH[:o, :o]) + np.einsum("ijij->", ERI[:o, :o, :o, :o]) / 2
    return F, E


def trans_t2(R, T1, T2, o):
    """TransT2 (PCCCI.f90:100-276): CI coefficients (C0, C1, C2) of the double similarity transform
    of 1 + T2 + T2^2/2 by V = [1 0; -T1 1] R, second order in the transformed T2."""
    M = R.shape[0]
    V = np.eye(M, dtype=complex)
    V[o:, :o] = -T1
    V = V @ R                                                        # :139-142
    U = np.zeros((M, M, M, M), dtype=complex)
    U[o:, o:, :o, :o] = T2
    U = int_tran4_sim(U, V)                                          # :143-145
    F, E0 = mkfock_mo(np.zeros((M, M), dtype=complex), U, o)        # :146 (0*V as the one-body part)
    C0 = 1.0 + E0                                                    # :148
    C1 = F[o:, :o].copy()                                            # :149
    C2 = U[o:, o:, :o, :o] / 4                                       # :150
    fov, fvo, foo, fvv = F[:o, o:], F[o:, :o], F[:o, :o], F[o:, o:]  # :153-156
    vvoo = U[o:, o:, :o, :o]
    oovv = U[:o, :o, o:, o:]
    C0 = C0 + E0 ** 2 / 2 + np.sum(fov * fvo.T) / 2                 # :161
    C0 = C0 + np.einsum("ijab,abij->", oovv / 8, vvoo, **ES)         # :162 tA_dot_tB
    C1 = C1 + E0 * fvo                                               # :163
    C1 = C1 - fvo @ foo / 2 + fvv @ fvo / 2                          # :164
    ooov = U[:o, :o, :o, o:]
    oovv = np.einsum("abij->ijab", vvoo)                             # :167 Transpose2(vvoo, oovv): the name
                                                                     # oovv now holds vvoo transposed
    C1 = C1 - np.einsum("ijab,ijkb->ak", oovv, ooov, **ES) / 4       # :168-174
    vvov = np.einsum("iabc->bcia", U[:o, o:, o:, o:])                # :178 vvov(b,c,i,a) = U(i,a,b,c)
    C1 = C1 - np.einsum("bcja,bckj->ak", vvov, vvoo, **ES) / 4       # :179-183
    ovov = U[:o, o:, :o, o:]                                         # :186
    C1 = C1 + np.einsum("abij,jb->ai", vvoo, fov, **ES) / 2          # :190
    C1 = C1 - np.einsum("jaib,bj->ai", ovov, fvo, **ES) / 2          # :191
    C2 = C2 + E0 / 4 * vvoo                                          # :196
    C2 = C2 - np.einsum("aj,bi->abij", fvo, fvo) / 2                 # :202
    C2 = C2 + np.einsum("jkac,kbic->abij", oovv, ovov, **ES) / 2     # :203
    C2tmp = np.zeros((o, o, M - o, M - o), dtype=complex)            # (i, j, a, b)
    vvvv = np.einsum("cdab->abcd", U[o:, o:, o:, o:])                # :213-214 Transpose1: vvvv(a,b,c,d) = U(c,d,a,b)
    C2tmp += np.einsum("cdij,cdab->ijab", vvoo / 16, vvvv, **ES)     # :215-221 (vvvv(c,d,a,b) = U(a,b,c,d))
    oooo = U[:o, :o, :o, :o]
    C2tmp += np.einsum("klij,klab->ijab", oooo / 16, oovv, **ES)     # :224-230
    C2tmp += np.einsum("ikab,kj->ijab", oovv, -foo / 4, **ES)        # :232-241
    C2tmp += np.einsum("ijcb,ac->ijab", oovv, fvv / 4, **ES)         # :243-249
    ooov = np.einsum("kaij->ijka", U[:o, o:, :o, :o])                # :252 ooov(i,j,k,a) = U(k,a,i,j)
    C2tmp += np.einsum("ijkb,ak->ijab", ooov, -fvo / 4, **ES)        # :253-259
    ovvv = np.einsum("abic->icab", U[o:, o:, :o, o:])                # :262 ovvv(i,c,a,b) = U(a,b,i,c)
    C2tmp += np.einsum("icab,cj->ijab", ovvv, fvo, **ES) / 4         # :263-271
    C2 = C2 + np.einsum("ijab->abij", C2tmp)                         # :274-275
    return C0, C1, C2


def asymm2(T2):
    """ASymm2 (CCRes.f90:31-70): X = T - T(ij swapped); T = X - X(ab swapped)."""
    X2 = T2 - np.einsum("abij->abji", T2)
    return X2 - np.einsum("abij->baij", X2)


def aperm(Mx, sort):
    """APerm (CCRes.f90:120-162): sort 1 antisymmetrises the first index pair, sort 2 the second."""
    if sort == 1:
        return Mx - np.einsum("ijab->jiab", Mx)
    return Mx - np.einsum("ijab->ijba", Mx)


def ci2cc(C0, C1, C2):
    """CI2CC (PCCCI.f90:72-98): T0 = C0, T1 = C1/C0, T2 = ASymm2(C2/C0 - T1 T1/2 for a != b, i != j).
    The a == b and i == j entries are zero after ASymm2 whether or not the product is subtracted
    there, so the product is subtracted everywhere."""
    T1 = C1 / C0
    T2 = C2 / C0 - np.einsum("ai,bj->abij", T1, T1) / 2
    return C0, T1, asymm2(T2)


def build_w(R, T1, T2, o):
    """BuildW (PCCCI.f90:14-40): TransT2 then CI2CC."""
    return ci2cc(*trans_t2(R, T1, T2, o))


def dstt2(R, T1, T2, o):
    """DSTT2 (FPUCC_Tools.f90:697-722): W0 = U0 W0', W1 = W1' + U1 with (U0, U1) = ProjT1(R, T1)
    and (W0', W1', W2) = BuildW(R, U1, T2)."""
    U0, U1 = proj_t1(R, T1, o)
    W0, W1, W2 = build_w(R, U1, T2, o)
    return W0 * U0, W1 + U1, W2


def cc_energy(T1, T2, Fock, ERI, o):
    """CCEnergy (CCRes.f90:9-29)."""
    e = np.sum(Fock[:o, o:] * T1.T)
    tau = T2 + np.einsum("ai,bj->abij", T1, T1) - np.einsum("bi,aj->abij", T1, T1)
    return e + np.einsum("ijab,abij->", ERI[:o, :o, o:, o:], tau, **ES) / 4


def cc_itms(Fock, H2, T1, T2, o):
    """CCItms (CCRes.f90:355-537): tau, Fvv, Foo, Fov, Woooo, Wvvvv, Wovvo."""
    Hoovv, Hooov, Hoovo = H2[:o, :o, o:, o:], H2[:o, :o, :o, o:], H2[:o, :o, o:, :o]
    itm1 = np.einsum("ai,bj->abij", T1, T1)                                   # :397-405
    itm4 = T2 / 2 + itm1                                                      # :407
    itm1 = np.einsum("abij->abij", itm1) - np.einsum("abij->baij", itm1)      # APerm(itm1, 1)
    itm1 = itm1 - np.einsum("abij->abji", itm1)                               # APerm(itm1, 2)
    tau = T2 + itm1 / 2                                                       # :410
    tb = T2 + itm1 / 4                                                        # :411
    Hvovv = H2[o:, :o, o:, o:]
    Fvv = Fock[o:, o:] - T1 @ Fock[:o, o:] / 2                                # :418
    Fvv = Fvv + np.einsum("ci,aibc->ab", T1, Hvovv, **ES)                     # :419-426
    Fvv = Fvv - np.einsum("abij,ijcb->ac", tb / 2, Hoovv, **ES)               # :428-433 (t2tmp = tb/2 transposed)
    Foo = Fock[:o, :o] + Fock[:o, o:] @ T1 / 2                                # :436
    Foo = Foo + np.einsum("ak,ikja->ij", T1, Hooov, **ES)                     # :437-443
    Foo = Foo + np.einsum("ikcb,cbjk->ij", Hoovv, tb / 2, **ES)               # :444-449
    Fov = Fock[:o, o:] + np.einsum("bj,ijab->ia", T1, Hoovv, **ES)            # :453-461
    Woooo = H2[:o, :o, :o, :o] + np.einsum("ijab,abkl->ijkl", Hoovv, tau / 4, **ES)   # :465-466
    itm2 = np.einsum("ijka,al->ijkl", Hooov, T1, **ES)                        # :469
    Woooo = Woooo + (itm2 - np.einsum("ijkl->ijlk", itm2))                    # :470-471 APerm(itm2, 2)
    Wvvvv = H2[o:, o:, o:, o:] + np.einsum("cdij,ijab->cdab", tau / 4, Hoovv, **ES)   # :474-480
    itm3 = np.einsum("aicd,bi->abcd", Hvovv, T1, **ES)                        # :482-494
    Wvvvv = Wvvvv - (itm3 - np.einsum("abcd->bacd", itm3))                    # :495-496 APerm(itm3, 1)
    Hovvv = H2[:o, o:, o:, o:]
    Wovvo = H2[:o, o:, o:, :o] + np.einsum("iabc,cj->iabj", Hovvv, T1, **ES)  # :502-509
    Wovvo = Wovvo - np.einsum("ikcj,bk->ibcj", Hoovo, T1, **ES)               # :510-517
    Wovvo = Wovvo - np.einsum("dbjk,ikcd->ibcj", itm4, Hoovv, **ES)           # :518-530
    return tau, Fvv, Foo, Fov, Woooo, Wvvvv, Wovvo


def cc_res12(Fock, H2, T1, T2, o):
    """CCRes12 (CCRes.f90:164-353): the CCSD residuals (res1 (v, o), res2 (v, v, o, o))."""
    tau, Fvv, Foo, Fov, Woooo, Wvvvv, Wovvo = cc_itms(Fock, H2, T1, T2, o)
    t2tmp = np.einsum("abij->ijab", T2)                                        # :206
    Hvoov, Hooov, Hvovv = H2[o:, :o, :o, o:], H2[:o, :o, :o, o:], H2[o:, :o, o:, o:]
    r1 = Fock[o:, :o] + Fvv @ T1 - T1 @ Foo                                   # :213
    r1 = r1 + np.einsum("jb,ijab->ai", Fov, t2tmp, **ES)                      # :217
    r1 = r1 + np.einsum("bj,ajib->ai", T1, Hvoov, **ES)                       # :218
    r1 = r1 - np.einsum("jkab,jkib->ai", t2tmp, Hooov, **ES) / 2              # :220-226
    r1 = r1 + np.einsum("ajcb,ijcb->ai", Hvovv, t2tmp, **ES) / 2              # :227-233
    r2 = H2[o:, o:, :o, :o]                                                   # :237
    itm1 = Fvv - T1 @ Fov / 2                                                 # :239
    itm2 = np.einsum("ijac,bc->ijab", t2tmp, itm1, **ES)                      # :242-249
    r2tmp = aperm(itm2, 2)                                                    # :250-251
    itm3 = Foo + Fov @ T1 / 2                                                 # :254
    itm2 = np.einsum("ikab,kj->ijab", t2tmp, itm3, **ES)                      # :255-264
    r2tmp = r2tmp - aperm(itm2, 1)                                            # :266-267
    Hvoov2 = np.einsum("iabj->bjia", H2[:o, o:, o:, :o])                      # :271 Hvoov(b,j,i,a) = H2(i,a,b,j)
    itm4 = np.einsum("ck,cjib->kjib", T1, Hvoov2, **ES)                       # :273-278 (o, o, o, v)
    itm2 = -np.einsum("kjib,ai->kjab", itm4, T1, **ES)                        # :280-286
    itm2 = itm2 + np.einsum("ikac,kbcj->ijab", t2tmp, Wovvo, **ES)            # :288-302
    itm2 = aperm(aperm(itm2, 1), 2)                                           # :304-305
    r2tmp = r2tmp + itm2                                                      # :306
    r2tmp = r2tmp + np.einsum("cdij,abcd->ijab", tau / 2, Wvvvv, **ES)        # :308-314 (Transpose1 of Wvvvv)
    r2tmp = r2tmp + np.einsum("klij,abkl->ijab", Woooo, tau / 2, **ES)        # :316-322
    Hvovv2 = np.einsum("abci->ciab", H2[o:, o:, o:, :o])                      # :327 Hvovv(c,i,a,b) = H2(a,b,c,i)
    Hooov2 = np.einsum("kaij->ijka", H2[:o, o:, :o, :o])                      # :328 Hooov(i,j,k,a) = H2(k,a,i,j)
    itm2 = np.einsum("ci,cjab->ijab", T1, Hvovv2, **ES)                       # :329-336
    r2tmp = r2tmp + aperm(itm2, 1)                                            # :337-338
    itm2 = np.einsum("ijkb,ak->ijab", Hooov2, T1, **ES)                       # :339-346
    r2tmp = r2tmp - aperm(itm2, 2)                                            # :347-348
    res2 = np.einsum("ijab->abij", r2tmp) + r2                                # :349-351
    return r1, res2


def _sz_masks(o, M):
    """Spin labels of the MO order [occ alpha, occ beta, vir alpha, vir beta] (NOA = o/2,
    NVA = M/2 - NOA) used by ProjSz1 / ProjSz2VO (FPUCC_Tools.f90:171-234)."""
    noa = o // 2
    nva = M // 2 - noa
    so = np.array([0] * noa + [1] * (o - noa))
    sv = np.array([0] * nva + [1] * (M - o - nva))
    m1 = sv[:, None] == so[None, :]
    m2 = (sv[:, None, None, None] + sv[None, :, None, None]) == (so[None, None, :, None] + so[None, None, None, :])
    # ProjSz2VO keeps aaaa, bbbb, abab, abba, baba, baab: exactly the Sz-conserving (a, b, i, j)
    return m1, m2


def proj_sz1(R1, o, M):
    """ProjSz1 on the vo block (FPUCC_Tools.f90:171-180)."""
    return np.where(_sz_masks(o, M)[0], R1, 0)


def proj_sz2_vo(R2, o, M):
    """ProjSz2VO (FPUCC_Tools.f90:217-234)."""
    return np.where(_sz_masks(o, M)[1], R2, 0)


def build_kern_sd(Fock, ERI, ESCF, U1t, U2t, o, SP):
    """BuildKernSD (FPUCC_Tools.f90:291-436), vo and vvoo blocks (the only ones EvalKernel keeps):
    Ovl1, Ovl2, EOvl0, EOvl1, EOvl2."""
    M = Fock.shape[0]
    Ovl1 = proj_sz1(U1t, o, M) if SP == 2 else U1t.copy()                              # :329-332
    Ovl2 = U2t + np.einsum("ai,bj->abij", U1t, U1t) - np.einsum("bi,aj->abij", U1t, U1t)  # :348-350
    if SP == 2:
        Ovl2 = proj_sz2_vo(Ovl2, o, M)                                                 # :356-358
    EOvl0 = cc_energy(U1t, U2t, Fock, ERI, o) + ESCF                                   # :361-362
    tmpEx1, tmpEx2 = cc_res12(Fock, ERI, U1t, U2t, o)                                  # :366
    EOvl1 = tmpEx1 + U1t * EOvl0                                                       # :392
    if SP == 2:
        EOvl1 = proj_sz1(EOvl1, o, M)                                                  # :398-400
    EOvl2 = (tmpEx2 + Ovl2 * EOvl0                                                     # :416-421
             + np.einsum("ai,bj->abij", U1t, tmpEx1) - np.einsum("bi,aj->abij", U1t, tmpEx1)
             + np.einsum("bj,ai->abij", U1t, tmpEx1) - np.einsum("aj,bi->abij", U1t, tmpEx1))
    if SP == 2:
        EOvl2 = proj_sz2_vo(EOvl2, o, M)                                               # :426-428
    return Ovl1, Ovl2, EOvl0, EOvl1, EOvl2


def ccsd_t_energy(F, H2, T1, T2, o):
    """CCSD_T_Ene (CCSD_T.f90:10-52) with get_wv (:54-70) and Perm3 (:72-88): the (T) energy of the
    amplitudes, a triangular loop a >= b >= c over virtual triples."""
    M = F.shape[0]
    v = M - o
    fvo = F[o:, :o]
    vvvo, ovoo, vvoo = H2[o:, o:, o:, :o], H2[:o, o:, :o, :o], H2[o:, o:, :o, :o]
    fd = np.diag(F)
    eijk = fd[:o, None, None] + fd[None, :o, None] + fd[None, None, :o]           # DirectSum3
    eabc = fd[o:, None, None] + fd[None, o:, None] + fd[None, None, o:]

    def get_wv(a, b, c):
        w = np.einsum("dk,dij->kij", vvvo[b, c], T2[a], **ES)                     # At_dot_B (:62)
        w = w - np.einsum("xl,lyz->xyz", T2[b, c], ovoo[:, a], **ES)             # A_dot_B (:63)
        vv = np.einsum("x,yz->xyz", T1[a], vvoo[b, c]) + np.einsum("x,yz->xyz", fvo[a], T2[b, c])  # A_outer_B
        vv = vv + w
        w = w + np.einsum("kij->ijk", w) + np.einsum("jki->ijk", w)              # Perm3: w + w(k,i,j) + w(j,k,i)
        return w, vv

    ene = 0j
    for a in range(v):
        for b in range(a + 1):
            for c in range(b + 1):
                wabc, vabc = get_wv(a, b, c)
                wcab, vcab = get_wv(c, a, b)
                wbac, vbac = get_wv(b, a, c)
                w = (wabc + wcab - wbac) / (eijk - eabc[a, b, c])
                ene += np.sum(w * np.conj(vabc + vcab - vbac))
    return ene / 2


def eval_kernel(HOne, HTwo, T1, T2, ENuc, RotMat, o, SP, TrunODE, fock=None):
    """EvalKernel (FPUCC.f90:529-602): the SD kernel for |TrunODE| 1 to 3, plus the (T) energy of the
    transformed amplitudes when TrunODE == 3 (:577-581).  Returns (eps0, lambda0, eps1, eps2, lambda1,
    lambda2)."""
    if abs(TrunODE) not in (1, 2, 3):
        raise ValueError("TrunODE 1, 2 or 3")
    M = HOne.shape[0]
    U0t, U1t, U2t = dstt2(RotMat, T1, T2, o)                                    # :561
    STot = U0t                                                                  # :565
    if fock is None:
        fock = mkfock_mo(HOne, HTwo, o)
    Fock, ESCF = fock                                                           # :566
    ESCF = ESCF + ENuc                                                          # :567
    Ovl1, Ovl2, eps0, EOvl1, EOvl2 = build_kern_sd(Fock, HTwo, ESCF, U1t, U2t, o, SP)   # :568-572
    if TrunODE == 3:                                                            # :577-581
        eps0 = eps0 + ccsd_t_energy(Fock, HTwo, U1t, U2t, o)
    lam1t, lam2t, eps1t, eps2t = Ovl1, Ovl2, EOvl1, EOvl2
    if SP == 2:                                                                 # :584-589
        lam1t, eps1t = proj_sz1(lam1t, o, M), proj_sz1(eps1t, o, M)
        lam2t, eps2t = proj_sz2_vo(lam2t, o, M), proj_sz2_vo(eps2t, o, M)
    lambda0 = STot                                                              # :590-596
    return eps0 * lambda0, lambda0, eps1t * lambda0, eps2t * lambda0, lam1t * lambda0, lam2t * lambda0


def point_weights(QJ, SP, NPoints, Npg, ncipg, Roota, Rootb, Rooty, Weightsp, Weightpg, fsp, fpg):
    """Per-point weight of PbarHbarOlap (FPUCC.f90:160-176) summed over the Wigner pairs (M, N)
    and point-group components (P, Q), in the loop order IPointA, IPointY, IPG."""
    nl, ny = NPoints
    w = np.zeros((nl, ny, Npg), dtype=complex)
    for ia in range(nl):
        for iy in range(ny):
            for ig in range(Npg):
                acc = 0j
                for m in range(-QJ, QJ + 1):
                    for n in range(-QJ, QJ + 1):
                        for p in range(ncipg):
                            for q in range(ncipg):
                                if SP == 2:
                                    wig = wigner(QJ, m, n, Roota[ia], Rootb[iy], Rooty[ia])
                                else:
                                    wig = wigner(QJ, m, n, Roota[ia], Rootb[ia], Rooty[iy])
                                wt = Weightsp[ia, iy] * Weightpg[ig, p, q]
                                wt = wig * wt * np.conj(fsp[QJ + m]) * fsp[QJ + n]
                                acc += wt * np.conj(fpg[p]) * fpg[q]
                w[ia, iy, ig] = acc
    return w.reshape(-1)


def pbarhbarolap(HOne, HTwo, T1, T2, NOcc, ENuc, QJ, SP, NPoints, Npg, ncik, R1, R2, Rpg, Rk, Roota, Rootb, Rooty,
                 Weightsp, Weightpg, fsp, fpg, fk, TrunODE, points=None):
    """PbarHbarOlap (FPUCC.f90:14-272).  ``points`` (flattened il, iy, ipg indices) restricts the sum
    to a subset of the grid, for checks at sizes where the whole grid is too slow here.
    Returns (Olap0, OlapEx1, OlapEx2, EOlap0, EOlapEx1, EOlapEx2)."""
    M = HOne.shape[0]
    o = NOcc
    v = M - o
    nl, ny = NPoints
    ncipg = Weightpg.shape[1]
    wts = point_weights(QJ, SP, NPoints, Npg, ncipg, Roota, Rootb, Rooty, Weightsp, Weightpg, fsp, fpg)
    acc = [0j, 0j, np.zeros((v, o), complex), np.zeros((v, o), complex), np.zeros((v, v, o, o), complex),
           np.zeros((v, v, o, o), complex)]  # EOlap0, Olap0, EOlapEx1, OlapEx1, EOlapEx2, OlapEx2
    sel = range(nl * ny * Npg) if points is None else points
    passes = [(HOne, HTwo, T1, T2, None, 1.0)]
    if ncik == 2:                                                                # :186-228
        passes.append((HOne.conj(), HTwo.conj(), T1.conj(), T2.conj(), Rk[1], fk[1]))
    for H1p, H2p, T1p, T2p, rk, fkw in passes:
        fock = mkfock_mo(H1p, H2p, o)
        for w in sel:
            ia, iy, ig = w // (ny * Npg), (w // Npg) % ny, w % Npg
            Rot = R1[ia] @ R2[iy] @ Rpg[ig]
            if rk is not None:
                Rot = Rot @ rk
            eps0, lam0, eps1, eps2, lam1, lam2 = eval_kernel(H1p, H2p, T1p, T2p, ENuc, Rot, o, SP, TrunODE, fock)
            wt = wts[w] * fkw
            for k, x in enumerate((eps0, lam0, eps1, lam1, eps2, lam2)):
                acc[k] = acc[k] + wt * x
    if SP == 2:                                                                  # :231-234 ProjSz
        for k in (2, 3):
            acc[k] = proj_sz1(acc[k], o, M)
        for k in (4, 5):
            acc[k] = proj_sz2_vo(acc[k], o, M)
    EOlap0, Olap0, EOlapEx1, OlapEx1, EOlapEx2, OlapEx2 = acc
    return Olap0, OlapEx1, OlapEx2, EOlap0, EOlapEx1, EOlapEx2


def pbarhbar_res_from_olap(Olap0, OlapEx1, OlapEx2, EOlap0, EOlapEx1, EOlapEx2, NOcc, NSO, SP):
    """PbarHbarResFromOlap (FPUCC.f90:394-427): Ene = EOlap0/Olap0, residuals (EOlapEx - Ene OlapEx)/Olap0."""
    Ene = EOlap0 / Olap0
    Res1 = (EOlapEx1 - Ene * OlapEx1) / Olap0
    Res2 = (EOlapEx2 - Ene * OlapEx2) / Olap0
    if SP == 2:
        Res1, Res2 = proj_sz1(Res1, NOcc, NSO), proj_sz2_vo(Res2, NOcc, NSO)
    return Ene, 0j, Res1, Res2


def make_pcc_problem(n, N, L, ngrid=(14, 8), seed=0, amp=0.05, spin_blocked=False, pg="None", SP=1, J=0):
    """The seeded projected-CC input of ``phf_pcc_b200.synth.make_pcc_problem`` (test data, not oracle
    arithmetic)."""
    from phf_pcc_b200 import synth

    return synth.make_pcc_problem(n, N, L, ngrid=ngrid, seed=seed, amp=amp, spin_blocked=spin_blocked, pg=pg,
                                  SP=SP, J=J)
