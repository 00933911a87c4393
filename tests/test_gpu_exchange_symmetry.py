"""The symmetric exchange form of the streamed J/K (exchange_symmetry).

For real integrals K(rho^T) = K(rho)^T, so the streamed form contracts the exchange rows of the index
pairs i <= k with the symmetric half of each density and those of the pairs i < k with the
antisymmetric half (half the exchange GEMM of the full rows), the Coulomb contraction runs over the
pairs l <= j, and each panel's Gram block keeps only the columns k >= i0.  Checked against the full
exchange rows of the same form (exchange_symmetry off) and against the spatial Cholesky C oracle:
FP64 (this library's GEMMs and cuBLAS) and the int8 slices, over panel schedules with ragged panels
(exchange_panel 1, 5 and automatic), n odd and n = 65 (the smallest n whose tensor-core plans slice
the densities apart from the density GEMM), and a grid split into several chunks (the last shorter).

Tolerances (relative to the largest element): FP64 forms 1e-11 against each other and 1e-10 against
the oracle; int8 slices (S = 5) 1e-9 against the FP64 forms.
"""
import numpy as np
import pytest

from oracle import phf_oracle as orc
from oracle import phf_oracle_c as corc
from phf_pcc_b200 import api, synth

pytestmark = pytest.mark.gpu


def _akw(p):
    kw = p.grid_kwargs()
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


def _err(a, b):
    return float(np.abs(a - b).max()) / max(1.0, float(np.abs(b).max()))


def _run(p, Ref, Z, **kw):
    with api.Plan(ref=Ref, h=p.h, B=p.B, jk_form="streamed", **_akw(p), **kw) as plan:
        return plan.buildhsg(Z, check_hermitian=False)


FORMS = [("fp64", dict(precision="fp64"), 1e-11), ("fp64 cublas", dict(precision="fp64", fp64_library_gemm=True), 1e-11),
         ("int8", dict(precision="ozaki_i8"), 1e-9)]


@pytest.mark.parametrize("n,N,L,panel", [(65, 6, 40, 5), (73, 9, 60, 1), (96, 10, 50, 0)])
def test_symmetric_exchange_matches_full_rows_and_oracle(n, N, L, panel):
    p = synth.make_problem(n, N, L, ngrid=(6, 3), seed=n + panel, pg="None")
    Ref, Z = p.ref_and_z()
    Z = Z + 0.05 * np.random.default_rng(n).normal(size=Z.shape)  # a non-Hermitian transition density
    kw = p.grid_kwargs()
    ora = corc.buildhsg(HOne=orc.mo_transform_1(p.hone_ao(), Ref), HTwo=None, Ref=Ref, Z=Z, Bs=p.B, **kw)
    full = _run(p, Ref, Z, precision="fp64", exchange_symmetry=False, exchange_panel=panel)
    for x, y in zip(full, ora):
        assert _err(x, y) <= 1e-10
    for label, fkw, tol in FORMS:
        sym = _run(p, Ref, Z, exchange_symmetry=True, exchange_panel=panel, **fkw)
        for x, y, key in zip(sym, full, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
            assert _err(x, y) <= tol, (label, key, _err(x, y))


def test_symmetric_exchange_over_chunks_matches_one_chunk():
    """A workspace that holds a few points splits the grid into chunks, the last one shorter: the
    density operands' column padding then differs between chunks."""
    p = synth.make_problem(70, 7, 30, ngrid=(6, 3), seed=4, pg="C2v")  # 72 points in blocks of 12
    Ref, Z = p.ref_and_z()
    one = _run(p, Ref, Z, precision="ozaki_i8")
    # ~1.63 MB of workspace per point at n = 70 (the int8 F X slices included): 80 MiB -> 48-point chunks
    with api.Plan(ref=Ref, h=p.h, B=p.B, jk_form="streamed", precision="ozaki_i8", workspace_bytes=80 << 20,
                  **_akw(p)) as plan:
        assert plan.chunk < 72 and 72 % plan.chunk != 0, plan.chunk  # 48-point chunks, the last of 24
        many = plan.buildhsg(Z, check_hermitian=False)
    for x, y in zip(many, one):
        assert _err(x, y) <= 1e-12


def test_symmetric_exchange_unavailable_for_fused_tensor_core_densities():
    p = synth.make_problem(40, 4, 20, ngrid=(6, 3), seed=1, pg="None")
    Ref, _ = p.ref_and_z()
    with pytest.raises(api.PHFError):
        api.Plan(ref=Ref, h=p.h, B=p.B, jk_form="streamed", precision="ozaki_i8", exchange_symmetry=True, **_akw(p))
