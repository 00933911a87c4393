"""GPU parity: the CUDA path (through the C ABI) against the golden vectors and the oracle.

Tolerances (FP64 on both sides, different summation orders):
  Hmat/Smat/Gradmat/Rdmmat: 1e-10 relative to the largest element
  energy: 1e-10 Eh; gradient elements G[N:, :N]: 1e-9
"""
import numpy as np
import pytest

from oracle import phf_oracle as orc
from phf_pcc_b200 import _lib, api, synth
from phf_pcc_b200.PHFTools_F import phftools
from tests._golden import CASES, grid_kwargs, htwo_mo, load

pytestmark = pytest.mark.gpu

REL = 1e-10


def _close(a, b, rel=REL):
    scale = max(1.0, float(np.abs(b).max()))
    return float(np.abs(np.asarray(a) - np.asarray(b)).max()) <= rel * scale


def _api_kwargs(c):
    k = grid_kwargs(c)
    return dict(ngrid=k["ngrid"], nci=k["nci"], cmplxconj=k["CmplxConj"], ncisp=k["ncisp"], nocc=k["NOcc"],
                r1=k["R1"], r2=k["R2"], rpg=k["Rpg"], weightsp=k["weightsp"], weightpg=k["weightpg"],
                roota=k["roota"], rootb=k["rootb"], rooty=k["rooty"], qj=k["QJ"], sp=k["SP"])


def _energy_grad(c, Hm, Sm, Gm, Rm):
    k = grid_kwargs(c)
    ncik = 2 if k["CmplxConj"] == 2 else 1
    e, v = orc.eigen_solver(Hm, Sm)
    fsp, fpg, fk = orc.vec_decomp(v[:, 0], k["ncisp"], k["ncipg"], ncik)
    G = api.localg(Gm, Rm, Sm, e[0], fsp, fpg, fk, k["CmplxConj"])
    N = int(c["N"])
    return e[0], G[N:, :N]


@pytest.mark.parametrize("name", CASES)
def test_dense_buildhsg_matches_golden(name):
    c = load(name)
    phftools.on_not_hermitian = "return"
    try:
        out = phftools.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], *[
            _api_kwargs(c)[k] for k in ("ngrid", "nci", "cmplxconj", "ncisp", "nocc", "r1", "r2", "rpg", "weightsp",
                                        "weightpg", "roota", "rootb", "rooty", "qj", "sp")], 0)
    finally:
        phftools.on_not_hermitian = "raise"
    for x, key in zip(out, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        assert x.flags.f_contiguous and x.dtype == np.complex128
        assert _close(x, c[key]), key
    e, G = _energy_grad(c, *out)
    assert abs(e - c["E0"]) <= 1e-10 * max(1.0, abs(c["E0"]))
    assert np.abs(G - c["G"]).max() <= 1e-9


@pytest.mark.parametrize("name", CASES)
def test_cholesky_buildhsg_fp64_matches_golden(name):
    c = load(name)
    out = api.buildhsg_chol(c["h"], c["B"], c["Ref"], c["Z"], check_hermitian=False, **_api_kwargs(c))
    for x, key in zip(out, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        assert _close(x, c[key]), key
    e, G = _energy_grad(c, *out)
    assert abs(e - c["E0"]) <= 1e-10 * max(1.0, abs(c["E0"]))
    assert np.abs(G - c["G"]).max() <= 1e-9


def test_not_hermitian_raises_like_the_reference_stop():
    c = load("tiny_sp1")  # coarse grid: the Fortran would STOP "Not Hermitian"
    with pytest.raises(_lib.PHFError) as ei:
        phftools.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], *[
            _api_kwargs(c)[k] for k in ("ngrid", "nci", "cmplxconj", "ncisp", "nocc", "r1", "r2", "rpg", "weightsp",
                                        "weightpg", "roota", "rootb", "rooty", "qj", "sp")], 0)
    assert ei.value.status == _lib.PHF_ERR_NOT_HERMITIAN


def test_localg_matches_oracle_cmplxconj2():
    c = load("cmplx2")
    k = grid_kwargs(c)
    e, v = orc.eigen_solver(c["Hmat"], c["Smat"])
    fsp, fpg, fk = orc.vec_decomp(v[:, 0], k["ncisp"], k["ncipg"], 2)
    G = api.localg(c["Gradmat"], c["Rdmmat"], c["Smat"], e[0], fsp, fpg, fk, 2)
    Go = orc.localg(c["Gradmat"], c["Rdmmat"], c["Smat"], e[0], fsp, fpg, fk, 2, k["NSO"], k["nci"], k["ncisp"],
                    k["ncipg"])
    assert np.abs(G - Go).max() <= 1e-12 * max(1.0, np.abs(Go).max())


def test_singular_overlap_reports_status():
    c = load("tiny_dense_htwo")
    kw = _api_kwargs(c)
    kw["r1"] = np.zeros_like(kw["r1"])  # R = 0 at every point: C^H R C = 0
    with pytest.raises(_lib.PHFError) as ei:
        api.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], **kw)
    assert ei.value.status == _lib.PHF_ERR_SINGULAR


def test_nonfinite_input_reports_status():
    c = load("tiny_dense_htwo")
    z = c["Z"].copy()
    z[0, 0] = np.nan
    with pytest.raises(_lib.PHFError) as ei:
        api.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], z, **_api_kwargs(c))
    assert ei.value.status == _lib.PHF_ERR_NONFINITE


def test_runs_are_bitwise_deterministic():
    c = load("c1")
    a = api.buildhsg_chol(c["h"], c["B"], c["Ref"], c["Z"], **_api_kwargs(c))
    b = api.buildhsg_chol(c["h"], c["B"], c["Ref"], c["Z"], **_api_kwargs(c))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_plan_reuse_and_chunking_agree():
    """A plan with a tiny workspace (many chunks) gives the one-shot result."""
    c = load("j1_c2v_b1")
    kw = _api_kwargs(c)
    ref = api.buildhsg_chol(c["h"], c["B"], c["Ref"], c["Z"], check_hermitian=False, **kw)
    with api.Plan(ref=c["Ref"], h=c["h"], B=c["B"], workspace_bytes=200_000, **kw) as plan:
        assert plan.chunk < 120
        for _ in range(2):
            out = plan.buildhsg(c["Z"], check_hermitian=False)
            for x, y in zip(out, ref):
                assert _close(x, y, 1e-12)


def test_midsize_cholesky_against_c_oracle_subset():
    """n = 32 (M = 64), N = 16, L = 96 with C2v on a reduced grid, against the C oracle."""
    from oracle import phf_oracle_c as corc

    p = synth.make_problem(32, 16, 96, ngrid=(6, 3), seed=5, pg="C2v")
    Ref, Z = p.ref_and_z()
    Z = 0.05 * (np.random.default_rng(1).normal(size=Z.shape) + 1j * np.random.default_rng(2).normal(size=Z.shape))
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    out = api.buildhsg_chol(p.h, p.B, Ref, Z, check_hermitian=False, **akw)
    Bt = np.transpose(orc.chol_spin_orbital(p.B, Ref), (1, 2, 0))
    H1 = orc.mo_transform_1(p.hone_ao(), Ref)
    ref = corc.buildhsg(H1, None, Ref, Z, Bt=Bt, **kw)
    for x, y, key in zip(out, ref, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        assert _close(x, y), key


def test_eval_device_matches_oracle():
    import torch

    c = load("tiny_sp1")
    kw = _api_kwargs(c)
    M, N = int(c["M"]), int(c["N"])
    newmo = np.vstack([np.eye(N), c["Z"]])
    C = c["Ref"] @ newmo                       # AO-basis determinant
    with api.Plan(ref=np.eye(M), h=c["h"], B=c["B"], **kw) as plan:
        hs, yg, yr = plan.eval_device(torch.from_numpy(C).cuda())
        hs, yg, yr = hs.cpu().numpy(), yg.cpu().numpy(), yr.cpu().numpy()
    # Gradmat_AO = Yg C^H; the golden Gradmat is Ref^H Gradmat_AO Ref
    G_mo = c["Ref"].conj().T @ (yg[0] @ C.conj().T) @ c["Ref"]
    R_mo = c["Ref"].conj().T @ (yr[0] @ C.conj().T) @ c["Ref"]
    assert _close(hs[0, 0], c["Hmat"][0, 0]) and _close(hs[0, 1], c["Smat"][0, 0])
    assert _close(G_mo, c["Gradmat"][0, 0]) and _close(R_mo, c["Rdmmat"][0, 0])


def test_point_range_plans_sum_to_the_full_grid():
    """The rank split: plans over disjoint point blocks add up to the full-grid sums."""
    import torch

    from phf_pcc_b200.distributed import point_range

    p = synth.make_problem(12, 6, 30, ngrid=(14, 5), seed=9, pg="C2v")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, **akw) as full:
        ref = [t.clone() for t in full.eval_device(C)]
    parts = []
    for r in range(3):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, point_range=point_range(p.grid.npoints, r, 3), **akw) as pl:
            parts.append([t.clone() for t in pl.eval_device(C)])
    for i in range(3):
        tot = parts[0][i] + parts[1][i] + parts[2][i]
        assert torch.allclose(tot, ref[i], rtol=0, atol=1e-12 * float(ref[i].abs().max()))


def test_graph_replay_matches_direct_launches():
    """eval_device replays a captured CUDA graph; with per-launch profiling on it launches kernel by
    kernel.  Both must give bitwise the same sums, call after call."""
    import torch

    p = synth.make_problem(16, 8, 40, ngrid=(6, 3), seed=4, pg="C2v")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    for prec in ("fp64", "ozaki_i8"):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=prec, workspace_bytes=400_000, **akw) as plan:
            graph = [[t.clone() for t in plan.eval_device(C)] for _ in range(2)]
            _lib.profile_enable(True)
            try:
                direct = [t.clone() for t in plan.eval_device(C)]
            finally:
                _lib.profile_enable(False)
        for a, b, c in zip(graph[0], graph[1], direct):
            assert torch.equal(a, b) and torch.equal(a, c)


@pytest.mark.parametrize("precision", ["fp64", "ozaki_i8"])
def test_spin_block_rotations_match_the_general_product(precision):
    """Spin rotations R1 are 2 x 2 block diagonal in the interleaved spin order, and a Cholesky plan
    then forms Y = R1 T2 from the blocks; a single extra entry of 1e-300 outside the blocks sends the
    same problem through the general M x M product.  Both must agree (the tiny entry changes the
    products by far less than the tolerance)."""
    import torch

    p = synth.make_problem(20, 10, 40, ngrid=(6, 3), seed=3, pg="C2v")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    res = []
    for tweak in (False, True):
        r1 = np.array(akw["r1"], dtype=np.complex128, copy=True)
        if tweak:
            r1[0, 0, p.M - 1] = 1e-300  # reference order: alpha orbital 0 -> beta orbital n - 1
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, jk_form="eri", precision=precision,
                      **dict(akw, r1=r1)) as plan:
            res.append([t.cpu().numpy() for t in plan.eval_device(C)])
    for a, b in zip(*res):
        assert _close(a, b, 1e-12), float(np.abs(a - b).max())
