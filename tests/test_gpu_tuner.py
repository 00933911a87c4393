"""The launch tuner (plans created with autotune): it times the candidate launch choices of every GEMM
shape a plan uses -- the FP64 GEMM's tile shape and the int8 GEMM's raster group -- at the plan's
first evaluation and keeps the fastest.  The candidates only reorder work, so a tuned plan must give
bitwise the results of an untuned one, in single evaluations, in buildhsg and in a batch."""
import numpy as np
import pytest

from phf_pcc_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu


def _akw(p):
    kw = p.grid_kwargs()
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


@pytest.mark.parametrize("precision,form", [("fp64", "eri"), ("ozaki_i8", "eri"), ("ozaki_i8", "streamed"),
                                            ("fp64", "factorized")])
def test_tuned_plans_are_bitwise_equal_to_untuned(precision, form):
    import torch

    p = synth.make_problem(24, 12, 60, ngrid=(14, 4), seed=31, pg="C2v")
    C = torch.from_numpy(p.C).cuda()
    Ref, Z = p.ref_and_z()
    res = {}
    before = int(_lib.load().phf_tuned_shapes())
    for tune in (False, True):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=precision, jk_form=form, autotune=tune,
                      exchange_panel=5, **_akw(p)) as plan:
            res[tune] = [[t.clone() for t in plan.eval_device(C)] for _ in range(2)]
        with api.Plan(ref=Ref, h=p.h, B=p.B, precision=precision, jk_form=form, autotune=tune, exchange_panel=5,
                      **_akw(p)) as plan:
            res[(tune, "bh")] = plan.buildhsg(Z, check_hermitian=False)
    assert int(_lib.load().phf_tuned_shapes()) > before or before > 0
    for a, b in zip(res[False][0], res[True][0]):
        assert torch.equal(a, b)
    for a, b in zip(res[True][0], res[True][1]):
        assert torch.equal(a, b)
    for a, b in zip(res[(False, "bh")], res[(True, "bh")]):
        assert np.array_equal(a, b)


def test_tuned_batch_equals_untuned_one_by_one():
    import torch

    probs = [synth.make_problem(n, n // 2, 3 * n, ngrid=(6, 3), seed=40 + n) for n in (16, 24, 16, 32)]
    Cs = [torch.from_numpy(p.C).cuda() for p in probs]
    ref = []
    for p, C in zip(probs, Cs):
        with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision="ozaki_i8", **_akw(p)) as plan:
            ref.append([t.clone() for t in plan.eval_device(C)])
    plans = [api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision="ozaki_i8", autotune=True, **_akw(p)) for p in probs]
    try:
        outs = api.eval_batch(plans, Cs)
        for o, r in zip(outs, ref):
            for a, b in zip(o, r):
                assert torch.equal(a, b)
    finally:
        for pl in plans:
            pl.close()
