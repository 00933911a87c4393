"""The int8 GEMM's wide issue (one MMA per A slice against the B slices it multiplies, laid side by
side in shared memory: 8 MMAs of up to 256 columns per k-block for 5 slices) against the narrow issue
(one 128 x BN x 32 MMA per slice pair, 15 for 5 slices).

Both forms add the same int8 products into the same exact int32 group sums and share the FP64
epilogue, so they must agree bit for bit: for every slice count the wide issue takes (1 to 5), on
ragged sizes (partial row and column tiles, k not a multiple of the 32-element k-block), on k long
enough for two launches whose second adds into D, in the split-k form, and through plans whose exchange
GEMM writes -K straight into Gamma."""
import numpy as np
import pytest

from phf_pcc_b200 import _lib, api, synth
from tests.test_gpu_ozaki import _bound_units, _dgemm

pytestmark = pytest.mark.gpu


class _wide:
    """Context manager: the wide issue on or off, restored on exit."""

    def __init__(self, on):
        self.on = on

    def __enter__(self):
        self.was = _lib.load().phf_int8_wide_mma(1 if self.on else 0)
        return self

    def __exit__(self, *exc):
        _lib.load().phf_int8_wide_mma(self.was)


@pytest.mark.parametrize("m,n,k,S", [(300, 200, 100, 5), (1000, 500, 3000, 5), (257, 96, 64, 4), (640, 130, 40, 3),
                                     (129, 97, 33, 1), (384, 256, 640, 2), (520, 300, 27000, 5)])
def test_wide_issue_matches_narrow_bitwise(m, n, k, S):
    rng = np.random.default_rng(m + 3 * n + 7 * k + S)
    A = rng.normal(size=(m, k)) * 10.0 ** rng.uniform(-3, 3, size=(m, 1))
    Bt = rng.normal(size=(n, k)) * 10.0 ** rng.uniform(-3, 3, size=(n, 1))
    with _wide(False):
        D1 = _dgemm(A, Bt, S)
    with _wide(True):
        D2 = _dgemm(A, Bt, S)
    assert np.array_equal(D1, D2), float(np.abs(D1 - D2).max())
    err = np.abs(D2 - A @ Bt.T) / _bound_units(A, Bt)
    assert err.max() <= 4.0 * (S + 1) * k * 2.0 ** (-7 * S), err.max()


def test_wide_setting_round_trips():
    lib = _lib.load()
    was = lib.phf_int8_wide_mma(0)
    try:
        assert lib.phf_int8_wide_mma(1) == 0
        assert lib.phf_int8_wide_mma(1) == 1
    finally:
        lib.phf_int8_wide_mma(was)


@pytest.mark.parametrize("form", ["streamed", "eri"])
def test_plan_results_identical_with_wide_and_narrow_issue(form):
    """Exchange GEMM into Gamma (row panels of the exchange matrix; the regeneration GEMM at a row
    offset of the Cholesky slices in the streamed form), split-k and plain Coulomb GEMMs: the whole
    evaluation is bitwise the same with either issue."""
    import torch

    p = synth.make_problem(40, 10, 60, ngrid=(6, 3), seed=9, pg="C2v")
    kw = p.grid_kwargs()
    akw = dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
               r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
               roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])
    C = torch.from_numpy(p.C).cuda()
    res = {}
    for on in (False, True):
        with _wide(on):
            with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, jk_form=form, precision="ozaki_i8", **akw) as plan:
                res[on] = [t.cpu().numpy() for t in plan.eval_device(C)]
    for a, b in zip(res[False], res[True]):
        assert np.array_equal(a, b), float(np.abs(a - b).max())
