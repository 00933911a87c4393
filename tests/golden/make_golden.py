"""Generate golden fixtures from the reference's own Python code.

Run in a container where the reference checkout is present:

    python tests/golden/make_golden.py /path/to/PHF_PCC

It imports the reference's PHFTools.py (per-grid-point Rdm, RdmConj, Kernels, Gradient,
LocalG, EigenSolver, VecDecomp), SpinSymm.py (RootWeight, RootWeightSy, BuildRotMat),
WignerMat.py, makeH.py (Mulliken2Dirac) and ao2mo.py (ao2mo), with stub modules in
place of ``parameter_fc``/``solve_ci``/``pyscf`` (which only carry module globals or are
absent here).  The grid-point loop is the BuildHSG order of PHF_fort/PHFTools.f90:84-170.
Outputs are written as compressed .npz files next to this script; the fixtures, not the
reference, are what the tests read.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _stub_modules(params: dict):
    pf = types.ModuleType("parameter_fc")
    for k, v in params.items():
        setattr(pf, k, v)
    sys.modules["parameter_fc"] = pf
    sys.modules["solve_ci"] = types.ModuleType("solve_ci")
    pyscf = types.ModuleType("pyscf")
    for sub in ("gto", "scf"):
        m = types.ModuleType("pyscf." + sub)
        setattr(pyscf, sub, m)
        sys.modules["pyscf." + sub] = m
    sys.modules["pyscf"] = pyscf


def _load_reference(ref_dir: str, params: dict):
    _stub_modules(params)
    for name in ("PHFTools", "SpinSymm", "WignerMat", "makeH", "ao2mo"):
        sys.modules.pop(name, None)
    if ref_dir not in sys.path:
        sys.path.insert(0, ref_dir)
    import PHFTools  # noqa: E402
    import SpinSymm  # noqa: E402
    import WignerMat  # noqa: E402
    import makeH  # noqa: E402
    import ao2mo  # noqa: E402
    return PHFTools, SpinSymm, WignerMat, makeH, ao2mo


def _hamiltonian(rng, n, L):
    h = rng.normal(size=(n, n)) * 0.1
    h = np.triu(h, 1)
    h = h + h.T
    h[np.diag_indices(n)] = np.linspace(-2.0, 0.0, n)
    A = rng.normal(scale=0.05, size=(L, n, n))
    B = np.triu(A) + np.transpose(np.triu(A, 1), (0, 2, 1))
    return h, B


def _unitary(rng, M):
    G = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    Q, _ = np.linalg.qr(G)
    return Q


def _reference_htwo(makeH, B, n):
    """Spin-orbital <ij||kl> as Main_PHF.py:22-30 does it (block copy + Mulliken2Dirac)."""
    M = 2 * n
    eri = np.einsum("Lpq,Lrs->pqrs", B, B)
    HTwo = np.zeros((M, M, M, M))
    HTwo[:n, :n, :n, :n] = eri
    HTwo[n:, n:, n:, n:] = eri
    HTwo[n:, n:, :n, :n] = eri
    HTwo[:n, :n, n:, n:] = eri
    return makeH.Mulliken2Dirac(HTwo)


def _c2v_ops(n, irrep):
    """Signed-diagonal C2v operations from round-robin labels (as PG_irrep.py:23-28)."""
    lab = np.arange(n) % 4
    ops = np.zeros((4, n, n))
    ops[0] = np.eye(n)
    ops[1] = np.diag((-1.0) ** (lab // 2))
    ops[2] = np.diag((-1.0) ** lab)
    ops[3] = ops[1] @ ops[2]
    ch = {"A1": (1, 1, 1, 1), "A2": (1, 1, -1, -1), "B1": (1, -1, 1, -1), "B2": (1, -1, -1, 1)}[irrep]
    wpg = np.array(ch, dtype=np.float64).reshape(4, 1, 1)
    Rpg = np.stack([np.kron(np.eye(2), ops[i]) for i in range(4)]).astype(np.complex128)
    return wpg, Rpg


def _c4v_ops(ref_dir, n, irrep):
    """The reference's C4vTable (PGSymm.py:109-137) -- its character or E-matrix weights -- with its
    pyscf-based orbital operations (SymmMat) replaced by synthetic block-diagonal ones that carry the
    C4v irreps (phf_pcc_b200.grid.c4v_orbital_ops), assembled as PG_Proj.py:21-25."""
    if ref_dir not in sys.path:
        sys.path.insert(0, ref_dir)
    sys.modules.pop("PGSymm", None)
    import PGSymm  # noqa: E402

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from phf_pcc_b200.grid import c4v_orbital_ops  # noqa: E402

    PGSymm.SymmMat = lambda pg, nrot, mol: c4v_orbital_ops(mol.nao)
    ID, nci, ops = PGSymm.C4vTable(types.SimpleNamespace(nao=n), irrep)
    weightpg = np.asarray(ID, dtype=np.float64)
    Rpg = np.stack([np.kron(np.eye(2), ops[i]) for i in range(ops.shape[0])]).astype(np.complex128)
    return weightpg, Rpg


def make_case(ref_dir, name, n, N, L, ngrid, seed, SP=1, J=0, CmplxConj=1, pg="None", irrep="A1",
              z_scale=0.1, store_htwo=False):
    M = 2 * n
    rng = np.random.default_rng(seed)
    h, B = _hamiltonian(rng, n, L)
    Ref = _unitary(rng, M)
    Z = z_scale * (rng.normal(size=(M - N, N)) + 1j * rng.normal(size=(M - N, N)))
    if CmplxConj == 0:
        Z = Z.real.astype(np.complex128)
    ncisp = 2 * J + 1 if SP == 1 else 1
    if pg == "C2v":
        weightpg, Rpg = _c2v_ops(n, irrep)
    elif pg == "C4v":
        weightpg, Rpg = _c4v_ops(ref_dir, n, irrep)
    else:
        weightpg, Rpg = np.ones((1, 1, 1)), np.eye(M, dtype=np.complex128)[None]
    npg = Rpg.shape[0]
    ncipg = weightpg.shape[1]
    ncik = 2 if CmplxConj == 2 else 1
    nci = ncisp * ncipg * ncik
    params = dict(NSO=M, NOccSO=N, ncisp=ncisp, ncipg=ncipg, ncik=ncik, CmplxConj=CmplxConj, SP=SP, J=J,
                  ngrid=list(ngrid), npg=npg)
    P, SS, WM, makeH, ao2mo = _load_reference(ref_dir, params)

    cwd = os.getcwd()
    os.chdir(ref_dir)  # RootWeight reads lebedev_*.txt relative to the working directory
    try:
        # Spin_Proj.py:3-39 logic, with the reference's own grid functions
        if SP == 1:
            roota, rootb, rooty, weightsp = SS.RootWeight(list(ngrid))
            R1 = np.stack([SS.BuildRotMat(roota[i], rootb[i], 0, n, M) for i in range(ngrid[0])])
            R2 = np.stack([SS.BuildRotMat(0, 0, rooty[i], n, M) for i in range(ngrid[1])])
        elif SP == 2:
            roota = rooty = np.zeros(1)
            rootb, wb = SS.RootWeightSy(ngrid[1])
            weightsp = wb[None, :].copy()
            R1 = np.eye(M, dtype=np.complex128)[None]
            R2 = np.stack([SS.BuildRotMat(0, rootb[i], 0, n, M) for i in range(ngrid[1])])
        elif SP == 3:
            roota, rootb, rooty, weightsp = SS.RootWeight(list(ngrid))
            R1 = np.zeros((ngrid[0], M, M), dtype=np.complex128)
            R1[0] = np.eye(M)
            R2 = np.stack([SS.BuildRotMat(0, 0, rooty[i], n, M) for i in range(ngrid[1])])
        else:
            raise ValueError(SP)
    finally:
        os.chdir(cwd)
    roota = np.asarray(roota, dtype=np.float64)
    rootb = np.asarray(rootb, dtype=np.float64)
    rooty = np.asarray(rooty, dtype=np.float64)

    HTwo_ao = _reference_htwo(makeH, B, n)
    HOne_ao = np.zeros((M, M))
    HOne_ao[:n, :n] = h
    HOne_ao[n:, n:] = h
    H1 = ao2mo.ao2mo(HOne_ao, Ref, 2)
    H2 = ao2mo.ao2mo(HTwo_ao, Ref, 4)

    # BuildHSG loop (PHFTools.f90:84-170) over the reference's per-point functions
    newMO = np.zeros((M, N), dtype=np.complex128)
    newMO[:N, :N] = np.eye(N)
    newMO[N:, :] = Z
    Hm = np.zeros((nci, nci), dtype=complex)
    Sm = np.zeros((nci, nci), dtype=complex)
    Gm = np.zeros((nci, nci, M, M), dtype=complex)
    Rm = np.zeros((nci, nci, M, M), dtype=complex)
    d = ncisp * ncipg
    for il in range(R1.shape[0]):
        for iy in range(R2.shape[0]):
            for ipg in range(npg):
                Rtmp = R1[il] @ R2[iy] @ Rpg[ipg]
                R = ao2mo.ao2mo(Rtmp, Ref, 2)
                rho0, s0 = P.Rdm(R, newMO)
                h0 = P.Kernels(H1, H2, rho0, s0)
                g0 = P.Gradient(H1, H2, rho0, s0)
                if CmplxConj == 2:
                    rho1, s1 = P.RdmConj(R, newMO)
                    h1 = P.Kernels(H1, H2, rho1, s1)
                    g1 = P.Gradient(H1, H2, rho1, s1)
                    rho0c, s0c = P.Rdm(R, newMO.conj())
                    g0c = P.Gradient(H1, H2, rho0c, s0c)
                    rho1c, s1c = P.RdmConj(R, newMO.conj())
                    g1c = P.Gradient(H1, H2, rho1c, s1c)
                else:
                    h1, g1, s1, rho1 = h0, g0, s0, rho0
                    g0c, s0c, rho0c = g0, s0, rho0
                    g1c, s1c, rho1c = g0, s0, rho0
                w0 = weightsp[il, iy]
                rho0, rho1 = rho0 * w0 * s0, rho1 * w0 * s1
                rho0c, rho1c = rho0c * w0 * s0c, rho1c * w0 * s1c
                h0, h1, s0, s1 = w0 * h0, w0 * h1, w0 * s0, w0 * s1
                g0, g1, g0c, g1c = g0 * w0, g1 * w0, g0c * w0, g1c * w0
                for ni in range(ncisp):
                    for nj in range(ncisp):
                        if SP == 2:
                            wig = WM.WignerMat(J, ni - J, nj - J, roota[il], rootb[iy], rooty[il])
                        else:
                            wig = WM.WignerMat(J, ni - J, nj - J, roota[il], rootb[il], rooty[iy])
                        for p in range(ncipg):
                            for q in range(ncipg):
                                w = weightpg[ipg, p, q] * wig
                                m = ni + p * ncisp
                                nn = nj + q * ncisp
                                Hm[m, nn] += h0 * w
                                Sm[m, nn] += s0 * w
                                Gm[m, nn] += g0 * w
                                Rm[m, nn] += rho0 * w
                                if CmplxConj == 2:
                                    Hm[m, nn + d] += h1 * w
                                    Sm[m, nn + d] += s1 * w
                                    Gm[m, nn + d] += g1 * w
                                    Rm[m, nn + d] += rho1 * w
                                    Gm[m + d, nn] += g1c * w
                                    Rm[m + d, nn] += rho1c * w
                                    Gm[m + d, nn + d] += g0c * w
                                    Rm[m + d, nn + d] += rho0c * w
    if CmplxConj == 2:
        Hm[d:, :d] = Hm[:d, d:].conj().T
        Sm[d:, :d] = Sm[:d, d:].conj().T
        Hm[d:, d:] = Hm[:d, :d]
        Sm[d:, d:] = Sm[:d, :d]
    evals, evecs = P.EigenSolver(Hm, Sm)
    fsp, fpg, fk = P.VecDecomp(evecs[:, 0])
    G = P.LocalG(Gm, Rm, Sm, evals[0], fsp, fpg, fk)      # (M-N, N) slice, PHFTools.py:176
    out = dict(n=n, N=N, L=L, M=M, ngrid=np.array(ngrid), SP=SP, J=J, CmplxConj=CmplxConj, npg=npg,
               ncisp=ncisp, ncipg=ncipg, nci=nci, h=h, B=B, Ref=Ref, Z=Z, R1=R1, R2=R2, Rpg=Rpg,
               weightsp=weightsp, weightpg=weightpg, roota=roota, rootb=rootb, rooty=rooty,
               Hmat=Hm, Smat=Sm, Gradmat=Gm, Rdmmat=Rm, E0=evals[0], evals=evals, fsp=fsp, fpg=fpg, fk=fk,
               G=G, HOne=H1)
    if store_htwo:
        out["HTwo"] = H2
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: E0={evals[0]!r}  nci={nci}  |Omega|={R1.shape[0] * R2.shape[0] * npg}  -> {path}")


def make_grid_fixture(ref_dir):
    _load_reference(ref_dir, dict(NSO=2, NOccSO=1, ncisp=1, ncipg=1, ncik=1, CmplxConj=1, SP=1, J=0))
    import SpinSymm as SS
    import WignerMat as WM
    cwd = os.getcwd()
    os.chdir(ref_dir)
    try:
        out = {}
        for ng in ((6, 4), (14, 8), (26, 3), (38, 2), (50, 16)):  # nl = 1 raises inside RootWeight (1-D loadtxt)
            a, b, y, w = SS.RootWeight(list(ng))
            key = f"rw_{ng[0]}_{ng[1]}"
            out[key + "_a"] = np.asarray(a)
            out[key + "_b"] = np.asarray(b)
            out[key + "_y"] = np.asarray(y, dtype=np.float64)
            out[key + "_w"] = np.asarray(w)
        for ny in (1, 4, 7):
            rb, wb = SS.RootWeightSy(ny)
            out[f"sy_{ny}_b"] = np.asarray(rb)
            out[f"sy_{ny}_w"] = np.asarray(wb)
        out["rot_args"] = np.array([[0.3, 1.1, 2.5], [1.0, 0.0, 0.0], [0.0, 2.0, 0.0], [-0.7, 0.4, 3.9]])
        out["rot"] = np.stack([SS.BuildRotMat(a, b, y, 3, 6) for a, b, y in out["rot_args"]])
        wig_args = []
        wig_vals = []
        for j in (0, 1, 2, 3):
            for n_ in range(-j, j + 1):
                for m_ in range(-j, j + 1):
                    for (al, be, ga) in ((0.3, 1.1, 2.5), (2.0, 2.9, -1.0)):
                        wig_args.append([j, n_, m_, al, be, ga])
                        wig_vals.append(WM.WignerMat(j, n_, m_, al, be, ga))
        out["wig_args"] = np.array(wig_args, dtype=np.float64)
        out["wig_vals"] = np.array(wig_vals, dtype=np.complex128)
    finally:
        os.chdir(cwd)
    path = os.path.join(HERE, "grids.npz")
    np.savez_compressed(path, **out)
    print("grids ->", path)


def main():
    ref_dir = os.path.abspath(sys.argv[1] if len(sys.argv) > 1 else "../PHF_PCC")
    make_grid_fixture(ref_dir)
    make_case(ref_dir, "tiny_sp1", n=5, N=3, L=7, ngrid=(6, 4), seed=11)
    make_case(ref_dir, "c1", n=20, N=10, L=120, ngrid=(14, 8), seed=1)
    make_case(ref_dir, "j1_c2v_b1", n=6, N=4, L=9, ngrid=(6, 5), seed=12, J=1, pg="C2v", irrep="B1")
    make_case(ref_dir, "j2_c2v_a1", n=5, N=4, L=5, ngrid=(14, 5), seed=15, J=2, pg="C2v", irrep="A1")
    make_case(ref_dir, "suhf_sp2_real", n=5, N=3, L=6, ngrid=(1, 6), seed=13, SP=2, CmplxConj=0)
    make_case(ref_dir, "cmplx2", n=4, N=2, L=5, ngrid=(6, 3), seed=14, CmplxConj=2)
    # SP = 3 is not generated: RootWeight fails for nl = 1 (1-D loadtxt), and for nl > 1
    # Spin_Proj.py:126 leaves R1[1:] = 0, which makes every overlap singular.
    make_case(ref_dir, "tiny_dense_htwo", n=3, N=2, L=4, ngrid=(6, 3), seed=17, store_htwo=True)
    # two-dimensional irrep (C4v E, ncipg = 2), alone and with J = 1 spin projection (nci = 6)
    make_case(ref_dir, "e_c4v", n=6, N=4, L=9, ngrid=(6, 4), seed=18, pg="C4v", irrep="E")
    make_case(ref_dir, "j1_e_c4v", n=5, N=3, L=6, ngrid=(6, 3), seed=19, J=1, pg="C4v", irrep="E")


if __name__ == "__main__":
    main()
