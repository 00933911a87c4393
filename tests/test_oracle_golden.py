"""The numpy oracle against golden vectors produced by the reference's own functions."""
import numpy as np
import pytest

from oracle import phf_oracle as orc
from tests._golden import CASES, grid_kwargs, htwo_mo, load


@pytest.mark.parametrize("name", CASES)
def test_buildhsg_dense_matches_reference(name):
    c = load(name)
    H2 = htwo_mo(c)
    Hm, Sm, Gm, Rm = orc.buildhsg(c["HOne"], H2, c["Ref"], c["Z"], **grid_kwargs(c))
    scale = max(1.0, np.abs(c["Hmat"]).max())
    assert np.abs(Hm - c["Hmat"]).max() <= 1e-11 * scale
    assert np.abs(Sm - c["Smat"]).max() <= 1e-12 * max(1.0, np.abs(c["Smat"]).max())
    assert np.abs(Gm - c["Gradmat"]).max() <= 1e-11 * max(1.0, np.abs(c["Gradmat"]).max())
    assert np.abs(Rm - c["Rdmmat"]).max() <= 1e-12 * max(1.0, np.abs(c["Rdmmat"]).max())


@pytest.mark.parametrize("name", CASES)
def test_energy_and_localg_match_reference(name):
    c = load(name)
    e, G, Hm, Sm = orc.energy_and_gradient(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], grid_kwargs(c))
    assert abs(e - c["E0"]) <= 1e-10 * max(1.0, abs(c["E0"]))
    N = int(c["N"])
    assert np.abs(G[N:, :N] - c["G"]).max() <= 1e-10


@pytest.mark.parametrize("name", ["tiny_sp1", "j1_c2v_b1", "cmplx2"])
def test_cholesky_gamma_equals_dense(name):
    c = load(name)
    Bso = orc.chol_spin_orbital(c["B"], c["Ref"])
    a = orc.buildhsg(c["HOne"], None, c["Ref"], c["Z"], Bso=Bso, **grid_kwargs(c))
    for x, key in zip(a, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        ref = c[key]
        assert np.abs(x - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max())


# Cases whose grids integrate exactly enough for the reference's Hermiticity check
# (PHFTools.f90:195-200); the Fortran would STOP "Not Hermitian" on the others.
HERMITIAN = {"c1": True, "cmplx2": True, "tiny_dense_htwo": True, "tiny_sp1": False, "j1_c2v_b1": False,
             "j2_c2v_a1": False, "suhf_sp2_real": False, "e_c4v": False, "j1_e_c4v": False}


@pytest.mark.parametrize("name", CASES)
def test_hermiticity_flag_on_golden(name):
    c = load(name)
    assert orc.hermiticity_violation(c["Hmat"], c["Smat"]) == (not HERMITIAN[name])


@pytest.mark.parametrize("name", CASES)
def test_c_oracle_matches_reference(name):
    from oracle import phf_oracle_c as corc
    c = load(name)
    kw = grid_kwargs(c)
    Hm, Sm, Gm, Rm = corc.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], **kw)
    for x, key in zip((Hm, Sm, Gm, Rm), ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        ref = c[key]
        assert np.abs(x - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), key
    e, v = orc.eigen_solver(Hm, Sm)
    ncik = 2 if kw["CmplxConj"] == 2 else 1
    fsp, fpg, fk = orc.vec_decomp(v[:, 0], kw["ncisp"], kw["ncipg"], ncik)
    G = corc.localg(Gm, Rm, Sm, e[0], fsp, fpg, fk, kw["CmplxConj"], kw["NSO"], kw["nci"], kw["ncisp"], kw["ncipg"])
    N = int(c["N"])
    assert np.abs(G[N:, :N] - c["G"]).max() <= 1e-10


@pytest.mark.parametrize("name", ["tiny_sp1", "cmplx2", "j1_c2v_b1"])
def test_c_oracle_cholesky_mode(name):
    from oracle import phf_oracle_c as corc
    c = load(name)
    Bso = orc.chol_spin_orbital(c["B"], c["Ref"])          # (L, M, M) MO basis
    Bt = np.transpose(Bso, (1, 2, 0))                       # (M, M, L)
    Hm, Sm, Gm, Rm = corc.buildhsg(c["HOne"], None, c["Ref"], c["Z"], Bt=Bt, **grid_kwargs(c))
    for x, key in zip((Hm, Sm, Gm, Rm), ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        ref = c[key]
        assert np.abs(x - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), key


@pytest.mark.parametrize("name", ["tiny_sp1", "cmplx2", "j1_c2v_b1", "c1"])
def test_c_oracle_spatial_cholesky_mode(name):
    """The spatial (AO-basis, real B_L) Cholesky form of the C oracle, with the grid points in
    parallel and with one point at a time split over the threads, against the golden vectors."""
    from oracle import phf_oracle_c as corc
    c = load(name)
    kw = grid_kwargs(c)
    npts = kw["ngrid"][0] * kw["ngrid"][1] * kw["npg"]
    sub = np.arange(0, npts, max(1, npts // 3))[:3]
    full = corc.buildhsg(c["HOne"], None, c["Ref"], c["Z"], Bs=c["B"], nthreads=2, **kw)
    for x, key in zip(full, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        ref = c[key]
        assert np.abs(x - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), key
    # a 3-point subset on 4 threads (one point at a time, split inside) against the MO-basis form
    Bt = np.transpose(orc.chol_spin_orbital(c["B"], c["Ref"]), (1, 2, 0))
    a = corc.buildhsg(c["HOne"], None, c["Ref"], c["Z"], Bs=c["B"], omega_list=sub, nthreads=4, **kw)
    b = corc.buildhsg(c["HOne"], None, c["Ref"], c["Z"], Bt=Bt, omega_list=sub, nthreads=1, **kw)
    for x, y in zip(a, b):
        assert np.abs(x - y).max() <= 1e-12 * max(1.0, np.abs(y).max())
