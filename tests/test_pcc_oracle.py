"""Checks of the projected-CC oracle (oracle/phf_pcc.py) against independent facts.

The reference's PCC kernel (SUCCSD_Boson_cmplx/FPUCC.f90) has no Python twin and its Fortran cannot
be built here, so the oracle is checked against quantities computed another way:

* the CCSD energy and residuals of CCEnergy / CCRes12 (CCRes.f90) against <Phi_mu| exp(-T) H exp(T)
  |Phi_0> evaluated with matrices in the space of all determinants (small M);
* ProjT1's Thouless factor against the determinant of the rotated occupied block;
* the identity rotation with T = 0: W0 = 1, W1 = W2 = 0, eps0 = E_SCF, residuals = H's vo / vvoo blocks.
"""
import itertools

import numpy as np
import pytest

from oracle import phf_pcc as pcc


def _fci_ops(M, o):
    """Determinants with o electrons in M spin orbitals, and a_p^dagger as matrices
    between the (o-1) -> o and o -> (o+1) electron spaces (Jordan-Wigner signs)."""
    def dets(k):
        return [frozenset(c) for c in itertools.combinations(range(M), k)]

    spaces = {k: dets(k) for k in range(max(0, o - 3), min(M, o + 3) + 1)}
    index = {k: {d: i for i, d in enumerate(v)} for k, v in spaces.items()}

    def create(p, k):  # a_p^dagger: space k -> k + 1
        A = np.zeros((len(spaces[k + 1]), len(spaces[k])))
        for j, d in enumerate(spaces[k]):
            if p in d:
                continue
            sign = (-1) ** sum(1 for q in d if q < p)
            A[index[k + 1][d | {p}], j] = sign
        return A

    return spaces, index, create


def _hbar_projections(h, H2, T1, T2, o):
    """<Phi_mu| e^-T H e^T |Phi_0> for mu = 0, singles (a, i), doubles (a, b, i, j), all in the
    o-electron space, with H = sum h_pq p^+ q + 1/4 sum <pq||rs> p^+ q^+ s r and
    T = sum t_ai a^+ i + 1/4 sum t_abij a^+ b^+ j i."""
    M = h.shape[0]
    spaces, index, create = _fci_ops(M, o)
    ad = {p: create(p, o - 1) for p in range(M)}       # (o-1) -> o
    ad2 = {p: create(p, o) for p in range(M)}          # o -> (o+1)
    ad0 = {p: create(p, o - 2) for p in range(M)}      # (o-2) -> (o-1)
    a = {p: ad[p].T for p in range(M)}                 # o -> (o-1)
    a0 = {p: ad0[p].T for p in range(M)}               # (o-1) -> (o-2)
    n = len(spaces[o])
    H = np.zeros((n, n), complex)
    for p in range(M):
        for q in range(M):
            if h[p, q] != 0:
                H += h[p, q] * (ad[p] @ a[q])
    for p, q, r, s in itertools.product(range(M), repeat=4):
        if H2[p, q, r, s] != 0:
            H += 0.25 * H2[p, q, r, s] * (ad[p] @ ad0[q] @ a0[s] @ a[r])
    v = M - o
    T = np.zeros((n, n), complex)
    for ai in range(v):
        for i in range(o):
            T += T1[ai, i] * (ad[o + ai] @ a[i])
    for ai, bi, i, j in itertools.product(range(v), range(v), range(o), range(o)):
        if T2[ai, bi, i, j] != 0:
            T += 0.25 * T2[ai, bi, i, j] * (ad[o + ai] @ ad0[o + bi] @ a0[j] @ a[i])
    del ad2
    from scipy.linalg import expm
    ref = np.zeros(n)
    ref[index[o][frozenset(range(o))]] = 1.0
    vec = expm(-T) @ H @ expm(T) @ ref
    e0 = vec @ ref
    r1 = np.zeros((v, o), complex)
    for ai in range(v):
        for i in range(o):
            phi = ad[o + ai] @ a[i] @ ref
            r1[ai, i] = phi @ vec
    r2 = np.zeros((v, v, o, o), complex)
    for ai, bi, i, j in itertools.product(range(v), range(v), range(o), range(o)):
        if ai == bi or i == j:
            continue
        phi = ad[o + ai] @ ad0[o + bi] @ a0[j] @ a[i] @ ref
        r2[ai, bi, i, j] = phi @ vec
    return e0, r1, r2


def _small_problem(M=8, o=4, seed=0):
    rng = np.random.default_rng(seed)
    h = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    h = 0.3 * (h + h.conj().T)
    g = rng.normal(size=(M, M, M, M)) + 1j * rng.normal(size=(M, M, M, M))
    g = g + np.einsum("pqrs->rspq", g).conj()          # <pq|rs> = <rs|pq>*
    g = g + np.einsum("pqrs->qpsr", g)                  # <pq|rs> = <qp|sr>
    H2 = 0.1 * (g - np.einsum("pqrs->pqsr", g))         # <pq||rs>
    v = M - o
    T1 = 0.1 * (rng.normal(size=(v, o)) + 1j * rng.normal(size=(v, o)))
    T2 = 0.1 * (rng.normal(size=(v, v, o, o)) + 1j * rng.normal(size=(v, v, o, o)))
    return h, H2, T1, pcc.asymm2(T2) / 4


def test_ccsd_residual_against_determinant_space():
    o = 4
    h, H2, T1, T2 = _small_problem(8, o)
    F, ESCF = pcc.mkfock_mo(h, H2, o)
    e_ref, r1_ref, r2_ref = _hbar_projections(h, H2, T1, T2, o)
    e = pcc.cc_energy(T1, T2, F, H2, o) + ESCF
    r1, r2 = pcc.cc_res12(F, H2, T1, T2, o)
    assert abs(e - e_ref) < 1e-10
    assert np.abs(r1 - r1_ref).max() < 1e-10
    assert np.abs(r2 - r2_ref).max() < 1e-10


def test_thouless_factor_is_occupied_determinant():
    rng = np.random.default_rng(3)
    M, o = 10, 4
    R = np.linalg.qr(rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M)))[0]
    T1 = 0.2 * (rng.normal(size=(M - o, o)) + 1j * rng.normal(size=(M - o, o)))
    U0, U1 = pcc.proj_t1(R, T1, o)
    Y = R[:, :o] + R[:, o:] @ T1
    assert abs(U0 - np.linalg.det(Y[:o])) < 1e-12
    # R [1; T1] = [1; U1] Y_occ: the rotated determinant in Thouless form
    assert np.abs(Y[o:] - U1 @ Y[:o]).max() < 1e-12


def test_identity_rotation_without_amplitudes():
    o = 4
    h, H2, _, _ = _small_problem(8, o, seed=1)
    M, v = 8, 4
    T1 = np.zeros((v, o), complex)
    T2 = np.zeros((v, v, o, o), complex)
    W0, W1, W2 = pcc.dstt2(np.eye(M, dtype=complex), T1, T2, o)
    assert abs(W0 - 1) < 1e-14 and np.abs(W1).max() == 0 and np.abs(W2).max() == 0
    eps0, lam0, eps1, eps2, lam1, lam2 = pcc.eval_kernel(h, H2, T1, T2, 0.0, np.eye(M, dtype=complex), o, 1, 1)
    F, ESCF = pcc.mkfock_mo(h, H2, o)
    assert abs(eps0 - ESCF) < 1e-12 and abs(lam0 - 1) < 1e-14
    assert np.abs(eps1 - F[o:, :o]).max() < 1e-12
    assert np.abs(eps2 - H2[o:, o:, :o, :o]).max() < 1e-12


def test_identity_rotation_keeps_amplitudes():
    """R = 1: the double similarity transform is exact to second order, so W = T for T1 = 0 and
    small T2 up to terms of third order in T2."""
    o = 4
    rng = np.random.default_rng(5)
    M, v = 8, 4
    T2 = 1e-3 * pcc.asymm2(rng.normal(size=(v, v, o, o)) + 1j * rng.normal(size=(v, v, o, o)))
    W0, W1, W2 = pcc.dstt2(np.eye(M, dtype=complex), np.zeros((v, o), complex), T2, o)
    assert abs(W0 - 1) < 1e-10
    assert np.abs(W1).max() < 1e-10
    assert np.abs(W2 - T2).max() < 1e-8


@pytest.mark.parametrize("sp", [1, 2])
def test_grid_kernel_small(sp):
    """A whole PbarHbarOlap pass on a small problem: finite, and the SP = 2 sums carry no
    spin-flip components."""
    prob = pcc.make_pcc_problem(4, 4, 12, ngrid=(6, 4) if sp == 1 else (2, 4), seed=2, spin_blocked=(sp == 2), SP=sp)
    prob.pop("MO")
    out = pcc.pbarhbarolap(**prob)
    assert all(np.all(np.isfinite(x)) for x in out)
    if sp == 2:
        o, M = prob["NOcc"], prob["HOne"].shape[0]
        m1, m2 = pcc._sz_masks(o, M)
        assert np.abs(out[1][~m1]).max() == 0 and np.abs(out[5][~m2]).max() == 0
