"""The int8-sliced tensor-core GEMM (phf_ozaki_dgemm) against FP64 products, and the
energy/gradient pipeline in that precision against the golden vectors.

Tolerances: slices are balanced base-254 digits in [-127, 127], so with S slices the dropped
products and the representation remainder are of order 254^{-S} < 2^{-7S}; an entry's error is
below (S+1) k 2^{-7S} max|A_i.| max|B_.j| (the test bound is 4x that).  Pipeline: |dE| <= 1e-9 Eh relative
to FP64, gradient elements <= 1e-8 (the benchmark target is 1e-8 Eh and 1e-7).
"""
import ctypes

import numpy as np
import pytest

from phf_pcc_b200 import _lib, api
from tests._golden import CASES, grid_kwargs, load

pytestmark = pytest.mark.gpu


def _dgemm(A, Bt, S):
    import torch

    dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(Bt)).cuda()
    m, k = A.shape
    n = Bt.shape[0]
    dD = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    st = _lib.load().phf_ozaki_dgemm(m, n, k, S, ctypes.c_void_p(dA.data_ptr()), k, ctypes.c_void_p(dB.data_ptr()),
                                     k, ctypes.c_void_p(dD.data_ptr()), n, ctypes.c_void_p(0))
    _lib.check(st, "phf_ozaki_dgemm")
    return dD.cpu().numpy()


def _bound_units(A, Bt):
    return np.abs(A).max(axis=1)[:, None] * np.abs(Bt).max(axis=1)[None, :]


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (200, 150, 333), (256, 192, 1000), (64, 40, 17)])
@pytest.mark.parametrize("S", [7, 6, 5, 3])
def test_ozaki_dgemm_matches_fp64(m, n, k, S):
    rng = np.random.default_rng(m * 7 + n * 3 + k + S)
    A = rng.normal(size=(m, k)) * 10.0 ** rng.uniform(-3, 3, size=(m, 1))
    Bt = rng.normal(size=(n, k)) * 10.0 ** rng.uniform(-3, 3, size=(n, 1))
    D = _dgemm(A, Bt, S)
    ref = A @ Bt.T
    err = np.abs(D - ref) / _bound_units(A, Bt)
    assert err.max() <= 4.0 * (S + 1) * k * 2.0 ** (-7 * S), err.max()
    if S == 3:  # the truncation is really there: 3 slices are far from FP64
        assert err.max() > 1e-12


def test_ozaki_dgemm_long_k_splits_into_exact_passes():
    rng = np.random.default_rng(5)
    A = rng.normal(size=(128, 30000))
    Bt = rng.normal(size=(64, 30000))
    D = _dgemm(A, Bt, 6)
    err = np.abs(D - A @ Bt.T) / _bound_units(A, Bt)
    assert err.max() <= 4.0 * 7 * 30000 * 2.0 ** -42


def _api_kwargs(c):
    k = grid_kwargs(c)
    return dict(ngrid=k["ngrid"], nci=k["nci"], cmplxconj=k["CmplxConj"], ncisp=k["ncisp"], nocc=k["NOcc"],
                r1=k["R1"], r2=k["R2"], rpg=k["Rpg"], weightsp=k["weightsp"], weightpg=k["weightpg"],
                roota=k["roota"], rootb=k["rootb"], rooty=k["rooty"], qj=k["QJ"], sp=k["SP"])


def _close(a, b, rel):
    return float(np.abs(a - b).max()) <= rel * max(1.0, float(np.abs(b).max()))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("form,precision", [("factorized", "fp64"), ("eri", "fp64"), ("eri", "fp64-cublas"),
                                            ("eri", "ozaki_i8"), ("streamed", "fp64"), ("streamed", "fp64-cublas"),
                                            ("streamed", "ozaki_i8"), ("streamed-3", "fp64"),
                                            ("streamed-3", "ozaki_i8")])
def test_forms_and_precisions_match_golden(name, form, precision):
    """Every J/K form and precision against the golden vectors.  "streamed-3": the exchange rows
    regenerated in panels of three spatial indices (c1, n = 20: six panels of 60 rows and one of 40)."""
    c = load(name)
    rel = 1e-10 if precision.startswith("fp64") else 1e-9
    lib_gemm = precision == "fp64-cublas"
    panel = int(form.split("-")[1]) if "-" in form else 0
    with api.Plan(ref=c["Ref"], h=c["h"], B=c["B"], jk_form=form.split("-")[0], precision=precision.split("-")[0],
                  fp64_library_gemm=lib_gemm, exchange_panel=panel, **_api_kwargs(c)) as plan:
        out = plan.buildhsg(c["Z"], check_hermitian=False)
    for x, key in zip(out, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        assert _close(x, c[key], rel), (key, float(np.abs(x - c[key]).max()))


@pytest.mark.parametrize("n,N,L", [(60, 21, 50), (64, 40, 64), (72, 10, 40)])
def test_int8_pipeline_matches_fp64_on_ragged_sizes(n, N, L):
    """n <= 64 forms and slices the density columns in one kernel (n = 60: n^2 not a multiple of the
    32-element k-block, N = 21 / 40 not multiples of the 16-column staging chunk); n = 72 takes the
    density GEMM followed by the column-slicing kernels.  Both must agree with the FP64 form."""
    import torch

    from phf_pcc_b200 import synth

    p = synth.make_problem(n, N, L, ngrid=(6, 3), seed=n + N, pg="C2v")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    res = {}
    for prec in ("fp64", "ozaki_i8"):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, jk_form="eri", precision=prec, **akw) as plan:
            res[prec] = [t.cpu().numpy() for t in plan.eval_device(C)]
    for a, b, what in zip(res["ozaki_i8"], res["fp64"], ("HS", "Yg", "Yr")):
        assert _close(a, b, 1e-9), (what, float(np.abs(a - b).max()))


@pytest.mark.parametrize("n", [130, 170])
def test_automatic_form_above_n128_streamed_matches_fp64_factorized(n):
    """Above n = 128 the automatic J/K form is the streamed one (no n^4 matrix; n = 130: panels of
    the 16900 x 16900 exchange matrix regenerated from the Cholesky vectors) in every precision; it
    must agree with the rank-N factorized FP64 form, which shares none of its exchange arithmetic.  The
    automatic streamed form uses the exchange symmetry (pairs i <= k and i < k, k = n(n+1)/2 and
    n(n-1)/2); the full exchange rows (exchange_symmetry off) are checked too: at n = 170 (k = n^2 =
    28900) each of their panels' exchange GEMMs needs two launches for exact int32 group sums, the
    second adding into Gamma."""
    import torch

    from phf_pcc_b200 import synth

    p = synth.make_problem(n, 4, 16, ngrid=(6, 3), seed=17, pg="None")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    res = {}
    for label, prec, form, sym in (("fact", "fp64", "factorized", "auto"), ("fp64", "fp64", "auto", "auto"),
                                   ("i8", "ozaki_i8", "auto", "auto"), ("fp64 full", "fp64", "auto", False),
                                   ("i8 full", "ozaki_i8", "auto", False)):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=prec, jk_form=form, exchange_symmetry=sym,
                      **akw) as plan:
            res[label] = [t.cpu().numpy() for t in plan.eval_device(C)]
        torch.cuda.empty_cache()
    for label, rel in (("fp64", 1e-11), ("i8", 1e-9), ("fp64 full", 1e-11), ("i8 full", 1e-9)):
        for a, b, what in zip(res[label], res["fact"], ("HS", "Yg", "Yr")):
            assert _close(a, b, rel), (label, what, float(np.abs(a - b).max()))
