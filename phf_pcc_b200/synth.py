"""Seeded synthetic PHF problems (orthonormal basis, S = I).

The reference reads molecular integrals from pyscf pickles; the workloads here are
synthetic stand-ins with the same shapes and value distributions:

* h   -- real symmetric n x n, off-diagonal N(0, 1) * 0.1, diagonal linspace(-2, 0, n)
* B_L -- real symmetric n x n with N(0, 0.05) entries (upper triangle mirrored);
         (pq|rs) = sum_L B_L[pq] B_L[rs] (8-fold symmetric, positive semidefinite)
* C   -- first N columns of the QR factor of an M x M complex Gaussian (M = 2n)

Spin orbitals are ordered [alpha block; beta block].  ``Problem.ref_and_z`` expresses C
in the reference's (Ref, Z) parameterisation (PHF.py:44, PHFTools.f90:69-77).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .grid import ProjectionGrid, make_grid

__all__ = ["Problem", "make_problem", "random_unitary", "orbital_rotation", "CONFIGS", "config_problem",
           "make_pcc_problem", "PCC_CONFIG"]


def random_unitary(M: int, rng: np.random.Generator) -> np.ndarray:
    G = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    Q, R = np.linalg.qr(G)
    return Q


def orbital_rotation(C: np.ndarray, scale: float, rng: np.random.Generator) -> np.ndarray:
    """C <- exp(kappa) C with kappa anti-Hermitian M x M, entries N(0, scale)."""
    M = C.shape[0]
    A = rng.normal(scale=scale, size=(M, M)) + 1j * rng.normal(scale=scale, size=(M, M))
    kappa = 0.5 * (A - A.conj().T)
    w, V = np.linalg.eigh(1j * kappa)            # 1j*kappa is Hermitian
    U = (V * np.exp(-1j * w)[None, :]) @ V.conj().T
    return U @ C


@dataclass
class Problem:
    n: int
    N: int
    L: int
    h: np.ndarray            # (n, n) real
    B: np.ndarray            # (L, n, n) real symmetric
    C: np.ndarray            # (M, N) complex, orthonormal columns
    grid: ProjectionGrid
    seed: int = 0
    Qfull: np.ndarray = field(default=None, repr=False)   # M x M unitary whose first N columns are C

    @property
    def M(self) -> int:
        return 2 * self.n

    def hone_ao(self) -> np.ndarray:
        M, n = self.M, self.n
        H = np.zeros((M, M), dtype=np.complex128)
        H[:n, :n] = self.h
        H[n:, n:] = self.h
        return H

    def ref_and_z(self):
        """(Ref, Z) with Ref unitary and Ref [I; Z] spanning the columns of C (Z = 0)."""
        M, N = self.M, self.N
        return self.Qfull.copy(), np.zeros((M - N, N), dtype=np.complex128)

    def grid_kwargs(self) -> dict:
        g = self.grid
        return dict(ngrid=list(g.ngrid), nci=g.nci, CmplxConj=g.CmplxConj, ncisp=g.ncisp, NOcc=self.N,
                    R1=g.R1, R2=g.R2, Rpg=g.Rpg, weightsp=g.weightsp, weightpg=g.weightpg,
                    roota=g.roota, rootb=g.rootb, rooty=g.rooty, QJ=g.J, SP=g.SP, npg=g.npg,
                    ncipg=g.ncipg, NSO=self.M)


def make_problem(n: int, N: int, L: int, ngrid=(14, 8), seed: int = 0, pg: str = "None", irrep: str = "A1",
                 SP: int = 1, J: int = 0, CmplxConj: int = 1) -> Problem:
    rng = np.random.default_rng(seed)
    h = rng.normal(size=(n, n)) * 0.1
    h = np.triu(h, 1)
    h = h + h.T
    h[np.diag_indices(n)] = np.linspace(-2.0, 0.0, n)
    A = rng.normal(scale=0.05, size=(L, n, n))
    B = np.triu(A) + np.transpose(np.triu(A, 1), (0, 2, 1))
    M = 2 * n
    Q = random_unitary(M, rng)
    C = Q[:, :N].copy()
    grid = make_grid(n, ngrid=ngrid, SP=SP, J=J, pg=pg, irrep=irrep, CmplxConj=CmplxConj)
    return Problem(n=n, N=N, L=L, h=h, B=B, C=C, grid=grid, seed=seed, Qfull=Q)


# The five workloads of the benchmark description (spatial n, electrons N, Cholesky L,
# grid, point group).  C4 (batched uneven instances) is generated by ``batch_problems``.
CONFIGS = {
    "c1": dict(n=20, N=10, L=120, ngrid=(14, 8), pg="None"),
    "c2": dict(n=64, N=32, L=400, ngrid=(50, 16), pg="C2v"),
    "c3": dict(n=128, N=64, L=800, ngrid=(50, 16), pg="None"),
    "c5": dict(n=200, N=100, L=1000, ngrid=(50, 16), pg="C2v"),
}


def config_problem(name: str, seed: int = 0) -> Problem:
    c = CONFIGS[name]
    return make_problem(c["n"], c["N"], c["L"], ngrid=c["ngrid"], seed=seed, pg=c["pg"])


def batch_problems(count: int = 256, seed: int = 0):
    """Uneven batch: n uniform in {16, 24, ..., 96}, N = n/2, L = 4n, grids [14,8] and
    [50,16] alternately (112 and 800 points)."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice(np.arange(16, 97, 8), size=count)
    out = []
    for i, n in enumerate(sizes):
        n = int(n)
        grid = (14, 8) if i % 2 == 0 else (50, 16)
        out.append(make_problem(n, n // 2, 4 * n, ngrid=grid, seed=seed * 100003 + i))
    return out


def _antisym_htwo(B):
    """Spin-orbital <ij||kl> from spatial Cholesky vectors (L, n, n): (pq|rs) = sum_L B_L[pq] B_L[rs] in the
    spin blocks of Main_PHF.py:22-29, then Mulliken -> Dirac with antisymmetrisation (makeH.py:63-67)."""
    n = B.shape[1]
    M = 2 * n
    eri = np.einsum("Lpq,Lrs->pqrs", B, B, optimize=True)
    Hm = np.zeros((M, M, M, M))
    a, b = slice(0, n), slice(n, M)
    for s1 in (a, b):
        for s2 in (a, b):
            Hm[s1, s1, s2, s2] = eri
    d = np.einsum("ijkl->ikjl", Hm)
    return d - np.einsum("ijkl->ijlk", d)


def make_pcc_problem(n, N, L, ngrid=(14, 8), seed=0, amp=0.05, spin_blocked=False, pg="None", SP=1, J=0):
    """Seeded projected-CC input (the arguments of PbarHbarOlap, SUCCSD_Boson_cmplx/FPUCC.f90:14-48) in an
    orthonormal MO basis: HOne, antisymmetrised HTwo, the grid rotations transformed to the MOs
    (MO^H R MO, as Main_PCC.py:35-40 does with ao2mo), and amplitudes T1 (v, o), T2 (v, v, o, o)
    antisymmetric with entries N(0, amp).  The Hamiltonian generator is ``make_problem``'s.

    ``spin_blocked``: MOs of definite spin in the order [occ alpha, occ beta, vir alpha, vir beta]
    (what the SP = 2 projection ProjSz assumes)."""
    p = make_problem(n, N, L, ngrid=ngrid, seed=seed, pg=pg, SP=SP, J=J)
    M = p.M
    rng = np.random.default_rng(seed + 7919)
    if spin_blocked:
        Qa = random_unitary(n, rng)
        Qb = random_unitary(n, rng)
        na = N // 2
        cols = [np.concatenate([Qa[:, :na], np.zeros((n, na))]),
                np.concatenate([np.zeros((n, N - na)), Qb[:, :N - na]]),
                np.concatenate([Qa[:, na:], np.zeros((n, n - na))]),
                np.concatenate([np.zeros((n, n - N + na)), Qb[:, N - na:]])]
        MO = np.concatenate(cols, axis=1)
    else:
        MO = p.Qfull
    Mc = MO.conj()
    H1 = Mc.T @ p.hone_ao() @ MO
    H2 = np.einsum("abcd,ai,bj,ck,dl->ijkl", _antisym_htwo(p.B), Mc, Mc, MO, MO, optimize=True)
    g = p.grid
    R1 = np.array([Mc.T @ r @ MO for r in g.R1])
    R2 = np.array([Mc.T @ r @ MO for r in g.R2])
    Rpg = np.array([Mc.T @ r @ MO for r in g.Rpg])
    v, o = M - N, N
    T1 = amp * (rng.normal(size=(v, o)) + 1j * rng.normal(size=(v, o)))
    T2 = amp * (rng.normal(size=(v, v, o, o)) + 1j * rng.normal(size=(v, v, o, o)))
    T2 = T2 - np.einsum("abij->abji", T2)
    T2 = (T2 - np.einsum("abij->baij", T2)) / 4
    return dict(HOne=H1, HTwo=H2, T1=T1, T2=T2, NOcc=N, ENuc=0.0, QJ=g.J, SP=g.SP,
                NPoints=(g.R1.shape[0], g.R2.shape[0]), Npg=g.npg, ncik=1, R1=R1, R2=R2, Rpg=Rpg,
                Rk=np.array([np.eye(M, dtype=complex)] * 2), Roota=g.roota, Rootb=g.rootb, Rooty=g.rooty,
                Weightsp=g.weightsp, Weightpg=g.weightpg, fsp=np.ones(g.ncisp, complex),
                fpg=np.ones(g.ncipg, complex), fk=np.ones(2, complex), TrunODE=1, MO=MO)


# The projected-CC grid workload: configuration 1's Hamiltonian generator and grid (n = 20, M = 40,
# N = 10, Lebedev 14 x 8 gamma = 112 points), CCSD-shaped amplitudes
PCC_CONFIG = dict(n=20, N=10, L=120, ngrid=(14, 8))
