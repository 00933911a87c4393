"""Batched evaluation of independent instances (phf_eval_batch) against one-by-one evaluation.

Instances of uneven size run as one CUDA graph spread over concurrent branches; every instance
must give bitwise the sums its own plan gives, on the first (capturing) call, on a replay, and
after the set changes (a plan destroyed: recapture)."""
import numpy as np
import pytest

from phf_pcc_b200 import api, synth

pytestmark = pytest.mark.gpu


def _kwargs(p):
    kw = p.grid_kwargs()
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


@pytest.mark.parametrize("precision", ["fp64", "ozaki_i8"])
def test_batch_matches_one_by_one(precision):
    import torch

    sizes = [8, 12, 16, 20, 24, 32, 40, 72, 16]  # includes n > 64 (unfused int8 operand path)
    probs = [synth.make_problem(n, n // 2, 3 * n, ngrid=((6, 3) if i % 2 else (14, 4)), seed=100 + i)
             for i, n in enumerate(sizes)]
    plans = [api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=precision, workspace_bytes=64 << 20, **_kwargs(p))
             for p in probs]
    try:
        Cs = [torch.from_numpy(p.C).cuda() for p in probs]
        ref = [[t.clone() for t in pl.eval_device(C)] for pl, C in zip(plans, Cs)]
        outs = api.eval_batch(plans, Cs)           # captures the batch graph
        outs = api.eval_batch(plans, Cs, outs)      # replays it
        for r, o in zip(ref, outs):
            for a, b in zip(r, o):
                assert torch.equal(a, b)
        # a changed set: the last plan destroyed, the rest evaluated again (recapture)
        plans[-1].close()
        outs2 = api.eval_batch(plans[:-1], Cs[:-1])
        for r, o in zip(ref[:-1], outs2):
            for a, b in zip(r, o):
                assert torch.equal(a, b)
    finally:
        for pl in plans:
            pl.close()
