"""The GPU-resident optimiser step (phf_pcc_b200.optimizer) against the reference's own optimiser run.

tests/golden/dropin_trace.npz holds five iterations of the reference's BFGS (PHF.py:23) on its own
EandG (PHF.py:55-91) for the c1 problem, started from z = 0, every function call recorded.  Here
the same scipy BFGS drives DeviceEandG (the dense Ref-MO Hamiltonian the driver passes, and the
Cholesky form in the AO basis): it must make the same calls with the same energies and gradients.
Then the device-resident L-BFGS loop runs from z = 0 with one host read per function evaluation;
its energies must decrease, and the oracle's energy at its final parameters must equal its own.

Tolerances: E within 1e-9 Eh and gradient elements within 1e-7 per call (FP64 on both sides; BFGS
carries the small differences from call to call), parameters within 1e-6.
"""
import os

import numpy as np
import pytest

from oracle import phf_oracle as orc
from phf_pcc_b200 import api
from phf_pcc_b200.optimizer import DeviceEandG, lbfgs, thouless_to_mos
from tests._golden import GOLDEN, grid_kwargs, htwo_mo, load

pytestmark = pytest.mark.gpu


def _akw(c):
    k = grid_kwargs(c)
    return dict(ngrid=k["ngrid"], nci=k["nci"], cmplxconj=k["CmplxConj"], ncisp=k["ncisp"], nocc=k["NOcc"],
                r1=k["R1"], r2=k["R2"], rpg=k["Rpg"], weightsp=k["weightsp"], weightpg=k["weightpg"],
                roota=k["roota"], rootb=k["rootb"], rooty=k["rooty"], qj=k["QJ"], sp=k["SP"])


def _plans(c):
    yield "mo", api.Plan(ref=c["Ref"], hone=c["HOne"], htwo=htwo_mo(c), **_akw(c))
    yield "ao", api.Plan(ref=c["Ref"], h=c["h"], B=c["B"], **_akw(c))


def test_reference_bfgs_trajectory_is_reproduced():
    from scipy.optimize import minimize

    c = load("c1")
    t = np.load(os.path.join(GOLDEN, "dropin_trace.npz"))
    M, N = int(c["M"]), int(c["N"])
    for basis, plan in _plans(c):
        with plan:
            de = DeviceEandG(plan, basis)
            calls = []

            def fun(x):
                E, g = de.host(x)
                calls.append((np.array(x), E, g))
                return E, g

            minimize(fun, np.zeros(2 * (M - N) * N), method="BFGS", jac=True, options={"gtol": 1e-4, "maxiter": 5})
        assert len(calls) == len(t["bfgs_E"]), (basis, len(calls))
        for k, (x, E, g) in enumerate(calls):
            assert np.abs(x - t["bfgs_x"][k]).max() <= 1e-6, (basis, k)
            assert abs(E - t["bfgs_E"][k]) <= 1e-9, (basis, k, E, t["bfgs_E"][k])
            assert np.abs(g - t["bfgs_g"][k]).max() <= 1e-7, (basis, k)


@pytest.mark.parametrize("precision", ["fp64", "ozaki_i8"])
def test_device_lbfgs_descends_with_one_host_read_per_evaluation(precision):
    import torch

    c = load("c1")
    M, N = int(c["M"]), int(c["N"])
    with api.Plan(ref=c["Ref"], h=c["h"], B=c["B"], precision=precision, **_akw(c)) as plan:
        de = DeviceEandG(plan, "ao")
        x0 = torch.zeros(2 * (M - N) * N, dtype=torch.float64, device="cuda")
        res = lbfgs(de, x0, maxiter=25, gtol=1e-4)
        assert res["host_reads"] == de.evaluations
        e = res["energies"]
        assert all(b <= a + 1e-12 for a, b in zip(e, e[1:])), e
        assert e[-1] < -24.8   # below the reference BFGS after five iterations (-24.89 there at iteration 5)
        x = res["x"].cpu().numpy()
    z = (x[:(M - N) * N] + 1j * x[(M - N) * N:]).reshape(M - N, N)
    eo, G, _, _ = orc.energy_and_gradient(c["HOne"], htwo_mo(c), c["Ref"], z, grid_kwargs(c))
    assert abs(eo - res["E"]) <= (1e-9 if precision == "fp64" else 1e-8), (eo, res["E"])
    g = res["g"].cpu().numpy()
    Gz = G[N:, :N]
    assert np.abs(np.concatenate([Gz.real.reshape(-1), Gz.imag.reshape(-1)]) - g).max() <= 1e-7


def test_thouless_to_mos_is_unitary_and_spans_the_determinant():
    import torch

    rng = np.random.default_rng(4)
    Z = 0.3 * (rng.normal(size=(7, 5)) + 1j * rng.normal(size=(7, 5)))
    U = thouless_to_mos(torch.from_numpy(Z).cuda()).cpu().numpy()
    assert np.allclose(U.conj().T @ U, np.eye(12), atol=1e-12)
    occ = np.vstack([np.eye(5), Z])
    # the first five columns span [I; Z]: projecting [I; Z] onto them loses nothing
    P = U[:, :5] @ U[:, :5].conj().T
    assert np.allclose(P @ occ, occ, atol=1e-12)
