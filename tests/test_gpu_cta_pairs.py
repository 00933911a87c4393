"""The int8 GEMM on CTA pairs (256-row tiles, tcgen05.mma.cta_group::2, each CTA of a cluster of two
holding its 128 rows of A and half of the B rows) against the same GEMM on single CTAs.

Every output element's group sums are exact int32 products in both forms and the FP64 epilogue is the
same code, so the two forms must agree bit for bit: on odd row-tile counts (the last pair's second
CTA reads rows past the matrix, which the loads fill with zeros and the epilogue does not store), on
k long enough for two launches whose second adds into D, for every single-pass slice count, and
through a plan whose exchange GEMM writes -K straight into Gamma."""
import ctypes

import numpy as np
import pytest

from phf_pcc_b200 import _lib, api, synth
from tests.test_gpu_ozaki import _bound_units, _dgemm

pytestmark = pytest.mark.gpu


class _pairs:
    """Context manager: the int8 GEMM's CTA pairs on or off, restored on exit."""

    def __init__(self, on):
        self.on = on

    def __enter__(self):
        self.was = _lib.load().phf_int8_cta_pairs(1 if self.on else 0)
        return self

    def __exit__(self, *exc):
        _lib.load().phf_int8_cta_pairs(self.was)


@pytest.mark.parametrize("m,n,k,S", [(300, 200, 100, 5), (1000, 500, 3000, 5), (257, 96, 64, 4), (640, 130, 40, 3),
                                     (129, 97, 33, 1), (384, 256, 640, 2), (520, 300, 27000, 5)])
def test_pairs_match_single_ctas_bitwise(m, n, k, S):
    rng = np.random.default_rng(m + 3 * n + 7 * k + S)
    A = rng.normal(size=(m, k)) * 10.0 ** rng.uniform(-3, 3, size=(m, 1))
    Bt = rng.normal(size=(n, k)) * 10.0 ** rng.uniform(-3, 3, size=(n, 1))
    with _pairs(False):
        D1 = _dgemm(A, Bt, S)
    with _pairs(True):
        D2 = _dgemm(A, Bt, S)
    assert np.array_equal(D1, D2), float(np.abs(D1 - D2).max())
    err = np.abs(D2 - A @ Bt.T) / _bound_units(A, Bt)
    assert err.max() <= 4.0 * (S + 1) * k * 2.0 ** (-7 * S), err.max()


def test_pair_setting_round_trips():
    lib = _lib.load()
    was = lib.phf_int8_cta_pairs(0)
    try:
        assert lib.phf_int8_cta_pairs(1) == 0
        assert lib.phf_int8_cta_pairs(1) == 1
    finally:
        lib.phf_int8_cta_pairs(was)


@pytest.mark.parametrize("form", ["streamed", "eri"])
def test_plan_results_identical_with_and_without_pairs(form):
    """Exchange GEMM into Gamma (row panels of the exchange matrix, the regeneration GEMM at a row
    offset of the Cholesky slices in the streamed form), Coulomb GEMMs: the whole evaluation is
    bitwise the same on CTA pairs and on single CTAs."""
    import torch

    p = synth.make_problem(40, 10, 60, ngrid=(6, 3), seed=9, pg="C2v")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    res = {}
    for on in (False, True):
        with _pairs(on):
            with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, jk_form=form, precision="ozaki_i8", **akw) as plan:
                res[on] = [t.cpu().numpy() for t in plan.eval_device(C)]
    for a, b in zip(res[False], res[True]):
        assert np.array_equal(a, b), float(np.abs(a - b).max())
