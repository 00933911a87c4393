"""Projection grids and projector data for the projected-HF grid kernel.

Host-side set-up, run once per calculation (O(|grid| * M^2)).  Everything here
produces the arrays that the reference passes to ``phftools.buildhsg``:

* ``root_weight``       -- SpinSymm.py:32-68  (Lebedev (alpha, beta) x trapezoid gamma)
* ``root_weight_sy``    -- SpinSymm.py:5-30   (Gauss-Legendre beta grid for SUHF)
* ``build_rot_mat``     -- SpinSymm.py:70-89  (spin-1/2 rotation as an M x M matrix)
* ``spin_proj``         -- Spin_Proj.py:3-39  (SP = 0/1/2/3 modes)
* ``wigner_D``          -- WignerMat.py:8-27 and PHF_fort/PHFTools.f90:350-376
* ``c2v_projector``     -- PG_irrep.py:6-28 (signed-diagonal C2v operations) with the
                           C2v characters of PGSymm.py:87-107, assembled as PG_Proj.py:17-26
* ``c4v_projector``     -- C4vTable (PGSymm.py:109-137): eight operations E, C4, C2, C4^3, sigma_xz,
                           sigma_yz, sigma_d, sigma_d' with the 1-D characters or, for the 2-D
                           irrep E (ncipg = 2), the 2 x 2 representation matrices as weights; the
                           orbital operations are block diagonal over synthetic orbital blocks
                           that carry the irreps of C4v (the reference takes them from pyscf AOs)
* ``no_pg``             -- PG_Proj.py:12-16

Spin-orbital order is [alpha block; beta block] (M = 2n), as BuildRotMat uses.

The Lebedev rules are built from their octahedral orbits (V. I. Lebedev, "Quadratures
on a sphere", USSR Comp. Math. Math. Phys. 16 (1976)); angles are returned in the
(phi, theta) convention of the reference's tables: phi = atan2(y, x) in degrees,
except at the poles where phi = 90 degrees, theta = acos(z).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = [
    "lebedev", "root_weight", "root_weight_sy", "build_rot_mat", "spin_rotation_2x2",
    "spin_proj", "wigner_D", "c2v_projector", "c4v_projector", "c4v_orbital_ops", "no_pg", "ProjectionGrid",
    "make_grid",
]

_SUPPORTED_NL = (1, 6, 14, 26, 38, 50)


def _orbit_a1():
    pts = []
    for ax in range(3):
        for s in (1.0, -1.0):
            v = [0.0, 0.0, 0.0]
            v[ax] = s
            pts.append(v)
    return pts


def _orbit_a2():
    a = 1.0 / math.sqrt(2.0)
    pts = []
    for zero_ax in range(3):
        for s1 in (1.0, -1.0):
            for s2 in (1.0, -1.0):
                v = []
                signs = [s1, s2]
                k = 0
                for ax in range(3):
                    if ax == zero_ax:
                        v.append(0.0)
                    else:
                        v.append(signs[k] * a)
                        k += 1
                pts.append(v)
    return pts


def _orbit_a3():
    a = 1.0 / math.sqrt(3.0)
    return [[sx * a, sy * a, sz * a] for sx in (1.0, -1.0) for sy in (1.0, -1.0) for sz in (1.0, -1.0)]


def _orbit_b(l):
    """24 points (l, l, m) and permutations/signs with 2 l^2 + m^2 = 1."""
    m = math.sqrt(1.0 - 2.0 * l * l)
    pts = []
    for m_ax in range(3):
        for s0 in (1.0, -1.0):
            for s1 in (1.0, -1.0):
                for s2 in (1.0, -1.0):
                    v = [0.0, 0.0, 0.0]
                    sg = [s0, s1, s2]
                    for ax in range(3):
                        v[ax] = sg[ax] * (m if ax == m_ax else l)
                    pts.append(v)
    return pts


def _orbit_c(p):
    """24 points (p, q, 0) and permutations/signs with p^2 + q^2 = 1."""
    q = math.sqrt(1.0 - p * p)
    pts = []
    for zero_ax in range(3):
        others = [ax for ax in range(3) if ax != zero_ax]
        for (u, w) in ((p, q), (q, p)):
            for s1 in (1.0, -1.0):
                for s2 in (1.0, -1.0):
                    v = [0.0, 0.0, 0.0]
                    v[others[0]] = s1 * u
                    v[others[1]] = s2 * w
                    pts.append(v)
    return pts


def _sphere_monomial_mean(a, b, c):
    """Average of x^a y^b z^c over the unit sphere (all exponents even)."""
    if a % 2 or b % 2 or c % 2:
        return 0.0
    # (a-1)!!(b-1)!!(c-1)!! / (a+b+c+1)!!
    def dfact(k):
        r = 1
        while k > 1:
            r *= k
            k -= 2
        return r
    return dfact(a - 1) * dfact(b - 1) * dfact(c - 1) / dfact(a + b + c + 1)


def _degree9_c_parameter():
    """Solve the c-orbit parameter of the 38-point (degree 9) rule.

    Weights 1/105 (a1), 9/280 (a3), 1/35 (c1) are fixed; p is fixed by exactness on
    x^4 y^4 (the first moment that the a1/a3 orbits alone do not satisfy)."""
    wa1, wa3, wc = 1.0 / 105.0, 9.0 / 280.0, 1.0 / 35.0
    target = _sphere_monomial_mean(4, 4, 0)

    def resid(p):
        s = 0.0
        for (pts, w) in ((_orbit_a1(), wa1), (_orbit_a3(), wa3), (_orbit_c(p), wc)):
            for x, y, z in pts:
                s += w * x ** 4 * y ** 4
        return s - target

    lo, hi = 0.75, 0.99  # bracket of the root with p > q
    flo = resid(lo)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        fm = resid(mid)
        if (fm > 0) == (flo > 0):
            lo, flo = mid, fm
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _lebedev_xyzw(nl):
    if nl == 1:
        return [[0.0, 0.0, 1.0]], [1.0]
    if nl == 6:
        orbits = [(_orbit_a1(), 1.0 / 6.0)]
    elif nl == 14:
        orbits = [(_orbit_a1(), 1.0 / 15.0), (_orbit_a3(), 3.0 / 40.0)]
    elif nl == 26:
        orbits = [(_orbit_a1(), 1.0 / 21.0), (_orbit_a2(), 4.0 / 105.0), (_orbit_a3(), 9.0 / 280.0)]
    elif nl == 38:
        orbits = [(_orbit_a1(), 1.0 / 105.0), (_orbit_a3(), 9.0 / 280.0),
                  (_orbit_c(_degree9_c_parameter()), 1.0 / 35.0)]
    elif nl == 50:
        orbits = [(_orbit_a1(), 4.0 / 315.0), (_orbit_a2(), 64.0 / 2835.0),
                  (_orbit_a3(), 27.0 / 1280.0), (_orbit_b(1.0 / math.sqrt(11.0)), 14641.0 / 725760.0)]
    else:
        raise ValueError(f"Lebedev grid with {nl} points is not supported; use one of {_SUPPORTED_NL}")
    pts, ws = [], []
    for o, w in orbits:
        pts.extend(o)
        ws.extend([w] * len(o))
    return pts, ws


def lebedev(nl: int):
    """Lebedev rule with ``nl`` points: (phi, theta, weight), angles in radians.

    Weights sum to 1 (the reference's tables, read by SpinSymm.py:47-63)."""
    if nl == 1:
        # single point at the north pole with phi = theta = 0 (lebedev_000 convention)
        return np.zeros(1), np.zeros(1), np.ones(1)
    pts, ws = _lebedev_xyzw(nl)
    phi = np.empty(nl)
    theta = np.empty(nl)
    for i, (x, y, z) in enumerate(pts):
        zc = max(-1.0, min(1.0, z))
        theta[i] = math.acos(zc)
        if abs(x) < 1e-15 and abs(y) < 1e-15:
            phi[i] = math.pi / 2.0
        else:
            phi[i] = math.atan2(y, x)
    return phi, theta, np.asarray(ws, dtype=np.float64)


def root_weight(ngrid):
    """Lebedev (alpha, beta) x trapezoid gamma grid (SpinSymm.py:32-68).

    gamma: ny points on [0, 2 pi] with spacing 2 pi/(ny-1) and halved end weights;
    weight[l, y] = w_lebedev[l] * w_gamma[y]."""
    nl, ny = int(ngrid[0]), int(ngrid[1])
    if ny == 1:
        rooty = np.zeros(1)
        weighty = np.ones(1)
    else:
        dx = 2.0 * math.pi / (ny - 1)
        rooty = np.arange(ny, dtype=np.float64) * dx
        weighty = np.full(ny, dx)
        weighty[0] = dx / 2.0
        weighty[-1] = dx / 2.0
    roota, rootb, wl = lebedev(nl)
    weight = np.outer(wl, weighty)
    return roota, rootb, rooty, weight


def root_weight_sy(ngrid: int):
    """Gauss-Legendre beta grid on [0, pi] times sin(beta) (SpinSymm.py:5-30).

    Nodes/weights by the Golub-Welsch eigenvalue method on the Legendre recurrence
    p_{k+1} = (2 - 1/(k+1)) x p_k - (1 - 1/(k+1)) p_{k-1}."""
    ngrid = int(ngrid)
    if ngrid == 1:
        return np.zeros(1), np.ones(1)
    k = np.arange(ngrid, dtype=np.float64)
    A = 2.0 - 1.0 / (k + 1.0)
    Cc = 1.0 - 1.0 / (k + 1.0)
    off = np.sqrt(Cc[1:] / (A[:-1] * A[1:]))
    T = np.diag(off, 1) + np.diag(off, -1)
    vals, vecs = np.linalg.eigh(T)
    w = 2.0 * vecs[0, :] ** 2
    rootb = (vals + 1.0) * math.pi / 2.0
    weightb = w * math.pi / 2.0 * np.sin(rootb)
    return rootb, weightb


def spin_rotation_2x2(a: float, b: float, y: float) -> np.ndarray:
    """2x2 spin-1/2 rotation diag(e^{ia/2}, e^{-ia/2}) [[cb, sb], [-sb, cb]] diag(e^{iy/2}, e^{-iy/2}).

    This is the spin factor U of BuildRotMat (SpinSymm.py:70-89): R = U (x) I_n."""
    ea = np.array([complex(math.cos(a / 2), math.sin(a / 2)), complex(math.cos(a / 2), -math.sin(a / 2))])
    ey = np.array([complex(math.cos(y / 2), math.sin(y / 2)), complex(math.cos(y / 2), -math.sin(y / 2))])
    cb, sb = math.cos(b / 2), math.sin(b / 2)
    Rb = np.array([[cb, sb], [-sb, cb]], dtype=np.complex128)
    return (ea[:, None] * Rb) * ey[None, :]


def build_rot_mat(a: float, b: float, y: float, n: int) -> np.ndarray:
    """M x M spin rotation (M = 2n) in [alpha; beta] order (SpinSymm.py:70-89)."""
    return np.kron(spin_rotation_2x2(a, b, y), np.eye(n))


def spin_proj(SP: int, ngrid, n: int, J: int = 0):
    """Spin-projection grid and rotation matrices (Spin_Proj.py:3-39).

    Returns (ncisp, roota, rootb, rooty, weights, R1, R2) with R1 (nl, M, M) and
    R2 (ny, M, M) complex."""
    M = 2 * n
    if SP == 0:
        eye = np.eye(M, dtype=np.complex128)[None]
        z = np.zeros(1)
        return 1, z, z.copy(), z.copy(), np.ones((1, 1)), eye.copy(), eye.copy()
    if SP == 1:
        roota, rootb, rooty, w = root_weight(ngrid)
        R1 = np.stack([build_rot_mat(roota[i], rootb[i], 0.0, n) for i in range(len(roota))])
        R2 = np.stack([build_rot_mat(0.0, 0.0, rooty[i], n) for i in range(len(rooty))])
        return 2 * J + 1, roota, rootb, rooty, w, R1, R2
    if SP == 2:
        rootb, wb = root_weight_sy(ngrid[1])
        z = np.zeros(1)
        w = wb[None, :].copy()
        R1 = np.eye(M, dtype=np.complex128)[None].copy()
        R2 = np.stack([build_rot_mat(0.0, rootb[i], 0.0, n) for i in range(len(rootb))])
        return 1, z, rootb, z.copy(), w, R1, R2
    if SP == 3:
        roota, rootb, rooty, w = root_weight(ngrid)
        # Spin_Proj.py:121-128 fills only R1[0]; the other Lebedev slots stay zero
        R1 = np.zeros((len(roota), M, M), dtype=np.complex128)
        R1[0] = np.eye(M)
        R2 = np.stack([build_rot_mat(0.0, 0.0, rooty[i], n) for i in range(len(rooty))])
        return 1, roota, rootb, rooty, w, R1, R2
    raise ValueError(f"unknown spin projection mode SP={SP}")


def wigner_D(j: int, n: int, m: int, alpha: float, beta: float, gamma: float) -> complex:
    """Wigner D^j_{nm}(alpha, beta, gamma) = e^{-i n alpha} d^j_{nm}(beta) e^{-i m gamma}.

    d^j_{nm} by the explicit factorial sum (WignerMat.py:8-27, PHFTools.f90:350-376)."""
    pre = math.sqrt(math.factorial(j + n) * math.factorial(j - n) * math.factorial(j + m) * math.factorial(j - m))
    smax = min(j + m, j - n)
    smin = max(0, m - n)
    acc = 0.0
    cb, sb = math.cos(beta / 2.0), math.sin(beta / 2.0)
    for s in range(smin, smax + 1):
        p1 = n - m + s
        p2 = 2 * j + m - n - 2 * s
        p3 = n - m + 2 * s
        num = (-1.0) ** p1 * cb ** p2 * sb ** p3
        den = math.factorial(j + m - s) * math.factorial(s) * math.factorial(n - m + s) * math.factorial(j - n - s)
        acc += num / den
    d = pre * acc
    return complex(np.exp(-1j * n * alpha) * d * np.exp(-1j * m * gamma))


_C2V_CHARACTERS = {
    # operations E, C2, sigma_xz, sigma_yz
    "A1": (1.0, 1.0, 1.0, 1.0),
    "A2": (1.0, 1.0, -1.0, -1.0),
    "B1": (1.0, -1.0, 1.0, -1.0),
    "B2": (1.0, -1.0, -1.0, 1.0),
}


def c2v_orbital_labels(n: int) -> np.ndarray:
    """Fixed round-robin C2v irrep labels (0..3 = A1, A2, B1, B2) for n spatial orbitals."""
    return np.arange(n, dtype=np.int64) % 4


def c2v_projector(n: int, irrep: str = "A1", labels=None):
    """C2v point-group projector data: (ncipg=1, weightpg (4,1,1), Rpg (4, M, M)).

    Operations are signed diagonals built from orbital irrep labels (PG_irrep.py:23-28):
    C2 = diag((-1)^(label // 2)), sigma_xz = diag((-1)^label), sigma_yz = C2 sigma_xz;
    Rpg[i] = blockdiag(op_i, op_i) (PG_Proj.py:21-25)."""
    if irrep not in _C2V_CHARACTERS:
        raise ValueError(f"unknown C2v irrep {irrep!r}")
    lab = c2v_orbital_labels(n) if labels is None else np.asarray(labels, dtype=np.int64)
    ops = np.zeros((4, n, n))
    ops[0] = np.eye(n)
    ops[1] = np.diag((-1.0) ** (lab // 2))
    ops[2] = np.diag((-1.0) ** lab)
    ops[3] = ops[1] @ ops[2]
    weightpg = np.array(_C2V_CHARACTERS[irrep], dtype=np.float64).reshape(4, 1, 1)
    Rpg = np.stack([np.kron(np.eye(2), ops[i]) for i in range(4)]).astype(np.complex128)
    return 1, weightpg, Rpg


# C4v in the operation order of PGSymm.py:109-137: E, C4, C2, C4^3, sigma_xz, sigma_yz, sigma_d, sigma_d'
_C4V_CHARACTERS = {
    "A1": (1.0,) * 8,
    "A2": (1.0, 1.0, 1.0, 1.0, -1.0, -1.0, -1.0, -1.0),
    "B1": (1.0, -1.0, 1.0, -1.0, 1.0, 1.0, -1.0, -1.0),
    "B2": (1.0, -1.0, 1.0, -1.0, -1.0, -1.0, 1.0, 1.0),
}


def c4v_e_matrices() -> np.ndarray:
    """The 2 x 2 matrices of the C4v irrep E in the operation order above: C4^k is the rotation by
    -k 90 degrees, and the reflections are rot(j) sigma_xz with j = 0, 2, 1, 3 for sigma_xz, sigma_yz,
    sigma_d, sigma_d' (sigma_xz = diag(1, -1)) -- the matrices of PGSymm.py:127-135."""
    def rot(k):
        c, s_ = round(math.cos(-k * math.pi / 2)), round(math.sin(-k * math.pi / 2))
        return np.array([[c, -s_], [s_, c]], dtype=np.float64)

    sxz = np.diag([1.0, -1.0])
    return np.stack([rot(0), rot(1), rot(2), rot(3)] + [rot(j) @ sxz for j in (0, 2, 1, 3)])


def c4v_orbital_ops(n: int) -> np.ndarray:
    """Eight n x n orbital operations of C4v (a representation of the group): orbitals fill blocks
    that transform as A1, E (a pair), B1, E, A2, B2, A1, ... in turn (a last single orbital that
    would start an E pair is A1)."""
    E2 = c4v_e_matrices()
    ops = np.zeros((8, n, n))
    kinds = ("A1", "E", "B1", "E", "A2", "B2")
    i = t = 0
    while i < n:
        kind = kinds[t % len(kinds)]
        t += 1
        if kind == "E" and i + 1 < n:
            ops[:, i:i + 2, i:i + 2] = E2
            i += 2
        else:
            ops[:, i, i] = _C4V_CHARACTERS["A1" if kind == "E" else kind]
            i += 1
    return ops


def c4v_projector(n: int, irrep: str = "A1"):
    """C4v point-group projector data (ncipg, weightpg (8, ncipg, ncipg), Rpg (8, M, M)) as
    C4vTable (PGSymm.py:109-137) and PG_Proj.py:17-26 assemble it: the weights are the irrep's
    characters, or the E matrices (ncipg = 2); Rpg[i] = blockdiag(op_i, op_i)."""
    if irrep == "E":
        ncipg, weightpg = 2, c4v_e_matrices()
    elif irrep in _C4V_CHARACTERS:
        ncipg, weightpg = 1, np.array(_C4V_CHARACTERS[irrep], dtype=np.float64).reshape(8, 1, 1)
    else:
        raise ValueError(f"unknown C4v irrep {irrep!r}")
    ops = c4v_orbital_ops(n)
    Rpg = np.stack([np.kron(np.eye(2), ops[i]) for i in range(8)]).astype(np.complex128)
    return ncipg, weightpg, Rpg


def no_pg(n: int):
    """Identity point group (PG_Proj.py:12-16): ncipg=1, weightpg=ones(1,1,1), Rpg=[I]."""
    M = 2 * n
    return 1, np.ones((1, 1, 1)), np.eye(M, dtype=np.complex128)[None].copy()


@dataclass
class ProjectionGrid:
    """All grid/projector arrays that ``buildhsg`` takes, plus the derived sizes."""
    SP: int
    ngrid: tuple
    J: int
    ncisp: int
    ncipg: int
    npg: int
    roota: np.ndarray
    rootb: np.ndarray
    rooty: np.ndarray
    weightsp: np.ndarray
    weightpg: np.ndarray
    R1: np.ndarray
    R2: np.ndarray
    Rpg: np.ndarray
    CmplxConj: int = 1

    @property
    def ncik(self) -> int:
        return 2 if self.CmplxConj == 2 else 1

    @property
    def nci(self) -> int:
        return self.ncisp * self.ncipg * self.ncik

    @property
    def npoints(self) -> int:
        return int(self.R1.shape[0] * self.R2.shape[0] * self.npg)


def make_grid(n: int, ngrid=(14, 8), SP: int = 1, J: int = 0, pg: str = "None", irrep: str = "A1",
              CmplxConj: int = 1) -> ProjectionGrid:
    """Build the spin (and optional C2v or C4v) projection grid for n spatial orbitals."""
    ncisp, roota, rootb, rooty, w, R1, R2 = spin_proj(SP, ngrid, n, J)
    if pg == "None":
        ncipg, wpg, Rpg = no_pg(n)
    elif pg == "C2v":
        ncipg, wpg, Rpg = c2v_projector(n, irrep)
    elif pg == "C4v":
        ncipg, wpg, Rpg = c4v_projector(n, irrep)
    else:
        raise ValueError(f"point group {pg!r} is not supported (None, C2v, C4v)")
    return ProjectionGrid(SP=SP, ngrid=tuple(int(g) for g in ngrid), J=J, ncisp=ncisp, ncipg=ncipg,
                          npg=Rpg.shape[0], roota=roota, rootb=rootb, rooty=rooty, weightsp=w,
                          weightpg=wpg, R1=R1, R2=R2, Rpg=Rpg, CmplxConj=CmplxConj)
