"""The drop-in module replays the reference driver's own calls (tests/golden/dropin_trace.npz).

The fixture was recorded by running the reference's unmodified ``EandG`` (PHF.py:55-91) twice on
the c1 problem (two optimiser steps) with a recording stand-in for the f2py module
(tests/golden/make_dropin_trace.py).  Here every recorded call goes, with the same positional
arguments, through ``from PHFTools_F import phftools`` -- the import line of PHF.py:10, resolved to
``dropin/PHFTools_F.py`` -- and its results must match the recorded ones.  The last check redoes
EandG's remaining arithmetic (EigenSolver of Hmat/Smat, the G[N:, :N] slice and the real/imaginary
concatenation of PHF.py:72-90) on the GPU results and compares with what the reference's EandG
returned.

Tolerances: Hmat/Smat/Gradmat/Rdmmat within 1e-10 of the largest element; E within 1e-10 Eh;
gradient vector within 1e-9.
"""
import os
import sys

import numpy as np
import pytest

from oracle import phf_oracle as orc
from tests._golden import GOLDEN, htwo_mo, load

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _dropin():
    path = os.path.join(ROOT, "dropin")
    if path not in sys.path:
        sys.path.insert(0, path)
    sys.modules.pop("PHFTools_F", None)
    from PHFTools_F import phftools  # noqa: E402  (the reference's import line)

    return phftools


def _calls():
    t = np.load(os.path.join(GOLDEN, "dropin_trace.npz"))
    c = load("c1")
    H2 = htwo_mo(c)
    calls = []
    for i in range(int(t["ncalls"])):
        args = []
        for j in range(int(t[f"call{i}_nargs"])):
            key = f"call{i}_arg{j}"
            if key + "_ref" in t.files:
                ref = str(t[key + "_ref"])
                args.append(H2 if ref == "HTwo" else c[ref])
            else:
                a = t[key]
                args.append(a.item() if a.ndim == 0 else a)
        calls.append((str(t[f"call{i}_name"]), args, i))
    return calls, t, c


def _close(a, b, rel):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max()) <= rel * max(1.0, float(np.abs(b).max()))


def test_dropin_module_is_the_library():
    from phf_pcc_b200.PHFTools_F import phftools as lib_phftools

    assert _dropin() is lib_phftools


def test_recorded_driver_calls_replay_through_the_dropin():
    phftools = _dropin()
    calls, t, c = _calls()
    outs = []
    for name, args, i in calls:
        if name == "buildhsg":
            res = phftools.buildhsg(*args)
            for x, k in zip(res, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
                assert x.flags.f_contiguous and x.dtype == np.complex128
                assert _close(x, t[f"call{i}_{k}"], 1e-10), (i, k)
        else:
            res = phftools.localg(*args)
            assert res.shape == t[f"call{i}_G"].shape
            assert _close(res, t[f"call{i}_G"], 1e-10), i
        outs.append(res)
    # EandG's remaining arithmetic on the GPU results (PHF.py:72-90, nci = 1, lamb = 0)
    N, M = int(c["N"]), int(c["M"])
    step = 0
    for k in range(0, len(calls), 2):
        Hm, Sm, Gm, Rm = outs[k]
        evals, evecs = orc.eigen_solver(Hm, Sm)
        fsp, fpg, fk = orc.vec_decomp(evecs[:, 0], 1, 1, 1)
        G = phftools.localg(Gm, Rm, Sm, evals[0], fsp, fpg, fk, 1, M, 1, 1, 1)[N:, :N].reshape(-1)
        g = np.concatenate([G.real, G.imag])
        assert abs(evals[0] - float(t[f"step{step}_E"])) <= 1e-10
        assert float(np.abs(g - t[f"step{step}_g"]).max()) <= 1e-9
        step += 1
    assert step == 2
