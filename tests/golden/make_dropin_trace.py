"""Record how the reference's own driver calls the f2py module, for the drop-in replay test.

Run in a container where the reference checkout is present:

    python tests/golden/make_dropin_trace.py /path/to/PHF_PCC

It imports the reference's unmodified PHF.py (with stub modules for ``parameter_fc``,
``solve_ci``, ``FixGauge`` and ``pyscf``, which only carry module globals or need absent
packages, and with ``PHFTools_F`` replaced by a recorder) and calls its ``EandG`` (PHF.py:55-91)
twice on the c1 golden problem (n = 20, M = 40, N = 10, Lebedev 14 x 8 grid): at the golden Z
and at a perturbed Z, as two optimiser steps would; then it runs five iterations of the BFGS
optimiser of PHF.py:23 on that EandG from z = 0 and records every function call (x, E, g).  The recorder's ``buildhsg`` and ``localg``
compute with the numpy oracle (itself pinned to the reference's functions by the golden tests)
and store every positional argument the driver passed and every result.  The fixture
``dropin_trace.npz`` holds, per call, the arguments (arrays that equal a field of c1.npz are
stored by that field's name; HTwo is rebuilt from c1's Cholesky vectors), the results, and
EandG's own returned (E, gradient vector), and the BFGS trajectory.  The replay test (tests/test_gpu_dropin.py) feeds the
same arguments to the drop-in module on the GPU.
"""
from __future__ import annotations

import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import phf_oracle as orc  # noqa: E402
from tests._golden import grid_kwargs, htwo_mo, load  # noqa: E402


class Recorder:
    """Stands in for the f2py module: records the driver's calls and answers with the oracle."""

    def __init__(self):
        self.calls = []

    def buildhsg(self, *args):
        (hone, htwo, ref, z, ngrid, nci, cc, ncisp, nocc, r1, r2, rpg, wsp, wpg, ra, rb, ry, qj, sp, comm, npg,
         ncipg, nso) = args
        out = orc.buildhsg(hone, htwo, ref, z, list(ngrid), nci, cc, ncisp, nocc, r1, r2, rpg, wsp, wpg, ra, rb, ry,
                           qj, sp, npg, ncipg, nso)
        self.calls.append(("buildhsg", args, out))
        return out

    def localg(self, *args):
        gm, rm, sm, e0, fsp, fpg, fk, cc, nso, nci, ncisp, ncipg = args
        G = orc.localg(gm, rm, sm, e0, fsp, fpg, fk, cc, nso, nci, ncisp, ncipg)
        self.calls.append(("localg", args, G))
        return G


def stub_modules(c):
    """Stand-ins for the reference's parameter module (the problem's globals), solve_ci, FixGauge and
    pyscf, none of which EandG computes with."""
    kw = grid_kwargs(c)
    n, M, N = int(c["n"]), int(c["M"]), int(c["N"])
    params = dict(NAO=n, NSO=M, NOccSO=N, NVrtSO=M - N, NOccA=N // 2, NVrtA=(M - N) // 2, NOccAO=N // 2,
                  ncisp=kw["ncisp"], ncipg=kw["ncipg"], ncik=1, nci=kw["nci"], CmplxConj=kw["CmplxConj"],
                  SP=kw["SP"], J=kw["QJ"], is_RHF=False, Enuc=0.0, ngrid=list(kw["ngrid"]), npg=kw["npg"],
                  R1=kw["R1"], R2=kw["R2"], Rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                  roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"])
    pf = types.ModuleType("parameter_fc")
    for k, v in params.items():
        setattr(pf, k, v)
    sys.modules["parameter_fc"] = pf
    sys.modules["solve_ci"] = types.ModuleType("solve_ci")
    fg = types.ModuleType("FixGauge")
    fg.FixGauge = lambda mos: mos
    fg.FixCmplxGauge = lambda f, mos: mos
    sys.modules["FixGauge"] = fg
    pyscf = types.ModuleType("pyscf")
    for sub in ("gto", "scf"):
        m = types.ModuleType("pyscf." + sub)
        setattr(pyscf, sub, m)
        sys.modules["pyscf." + sub] = m
    sys.modules["pyscf"] = pyscf


def main():
    ref_dir = os.path.abspath(sys.argv[1] if len(sys.argv) > 1 else "../PHF_PCC")
    c = load("c1")
    stub_modules(c)
    rec = Recorder()
    f2py = types.ModuleType("PHFTools_F")
    f2py.phftools = rec
    sys.modules["PHFTools_F"] = f2py
    sys.path.insert(0, ref_dir)
    HTwo = htwo_mo(c)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)  # EandG writes newsol.p and PHFout into the working directory
        try:
            import PHF  # noqa: E402  (the reference driver, unmodified)

            z0 = c["Z"].reshape(-1)
            rng = np.random.default_rng(3)
            z1 = z0 + 0.01 * (rng.normal(size=z0.shape) + 1j * rng.normal(size=z0.shape))
            results = []
            for z in (z0, z1):
                x = np.concatenate([z.real, z.imag])
                E, g = PHF.EandG(x, c["HOne"], HTwo, c["Ref"], 0)
                results.append((x, E, g))
            ncalls_eandg = len(rec.calls)
            # the reference's optimiser on its EandG (PHF.py:23's BFGS, started from z = 0 as optPHF
            # does without a saved solution), five iterations; every function call recorded
            from scipy.optimize import minimize

            traj = []

            def fun(x, *args):
                E, g = PHF.EandG(x, *args)
                traj.append((np.array(x), E, np.array(g)))
                return E, g

            M, N = int(c["M"]), int(c["N"])
            minimize(fun, np.zeros(2 * (M - N) * N), args=(c["HOne"], HTwo, c["Ref"], 0), method="BFGS", jac=True,
                     options={"gtol": 1e-4, "maxiter": 5})
            del rec.calls[ncalls_eandg:]
        finally:
            os.chdir(cwd)
    out = {"ncalls": len(rec.calls)}
    for i, (name, args, res) in enumerate(rec.calls):
        out[f"call{i}_name"] = name
        out[f"call{i}_nargs"] = len(args)
        for j, a in enumerate(args):
            key = f"call{i}_arg{j}"
            if a is HTwo:
                out[key + "_ref"] = "HTwo"
                continue
            hit = None
            if isinstance(a, np.ndarray):
                for fld in c:
                    if isinstance(c[fld], np.ndarray) and c[fld].shape == a.shape and c[fld].dtype == a.dtype \
                            and np.array_equal(c[fld], a):
                        hit = fld
                        break
            if hit is not None:
                out[key + "_ref"] = hit
            else:
                out[key] = np.asarray(a)
        if name == "buildhsg":
            for k, r in zip(("Hmat", "Smat", "Gradmat", "Rdmmat"), res):
                out[f"call{i}_{k}"] = r
        else:
            out[f"call{i}_G"] = res
    for s, (x, E, g) in enumerate(results):
        out[f"step{s}_x"] = x
        out[f"step{s}_E"] = E
        out[f"step{s}_g"] = g
    out["bfgs_x"] = np.array([t[0] for t in traj])
    out["bfgs_E"] = np.array([t[1] for t in traj])
    out["bfgs_g"] = np.array([t[2] for t in traj])
    path = os.path.join(HERE, "dropin_trace.npz")
    np.savez_compressed(path, **out)
    print(f"{len(rec.calls)} calls, E = {[r[1] for r in results]} -> {path}")


if __name__ == "__main__":
    main()
