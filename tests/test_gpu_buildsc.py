"""BuildSC on the GPU (phf_buildsc through the C ABI and phftools.buildsc) against the oracle.

Grids with C2v or the two-dimensional C4v irrep E and spin-projection channels (J = 1), random
complex vectors.  Tolerance: 1e-11 of the largest element of each output (FP64 on both sides)."""
import numpy as np
import pytest

from oracle.phf_buildsc import buildsc as buildsc_oracle
from phf_pcc_b200 import api, synth
from phf_pcc_b200.PHFTools_F import phftools

pytestmark = pytest.mark.gpu


def _case(n, N, seed, pg, irrep="A1", J=0, chunk_bytes=0):
    p = synth.make_problem(n, N, 4, ngrid=(6, 3), seed=seed, pg=pg, irrep=irrep, J=J)
    g = p.grid
    rng = np.random.default_rng(seed)
    M = p.M
    cz = lambda *s: rng.normal(size=s) + 1j * rng.normal(size=s)
    fsp = cz(g.ncisp) if g.ncisp > 1 else np.ones(1, complex)
    fpg = cz(g.ncipg) if g.ncipg > 1 else np.ones(1, complex)
    vec = (complex(cz(1)[0]), 0.3 * cz(M, M), 0.1 * cz(M, M, M, M))
    U = p.Qfull  # rotations in an MO basis (as LinDep.py passes them), so the projection is generic
    mo = lambda R: np.einsum("ai,gab,bj->gij", U.conj(), R, U)
    args = dict(nocc=N, ngrid=g.ngrid, qj=g.J, r1=mo(g.R1), r2=mo(g.R2), rpg=mo(g.Rpg), roota=g.roota,
                rootb=g.rootb, rooty=g.rooty, weightsp=g.weightsp, weightpg=g.weightpg, fsp=fsp, fpg=fpg)
    return vec, args, M


@pytest.mark.parametrize("n,N,seed,pg,irrep,J", [(3, 2, 1, "C2v", "A1", 0), (4, 3, 2, "C4v", "E", 0),
                                                 (3, 2, 3, "None", "A1", 1), (5, 4, 4, "C2v", "B1", 0)])
def test_buildsc_matches_oracle(n, N, seed, pg, irrep, J):
    vec, args, M = _case(n, N, seed, pg, irrep, J)
    ref = buildsc_oracle(*vec, **args)
    rk = np.eye(M, dtype=complex)[None]
    out = phftools.buildsc(*vec, args["nocc"], args["ngrid"], args["qj"], args["r1"], args["r2"], args["rpg"], rk,
                           args["roota"], args["rootb"], args["rooty"], args["weightsp"], args["weightpg"],
                           args["fsp"], args["fpg"], [1.0])
    assert out[1].flags.f_contiguous and out[2].flags.f_contiguous
    for x, y in zip(out, ref):
        x, y = np.asarray(x), np.asarray(y)
        assert np.abs(x - y).max() <= 1e-11 * max(1.0, float(np.abs(y).max())), float(np.abs(x - y).max())


def test_buildsc_singular_rotation_reports_status():
    vec, args, M = _case(3, 2, 5, "None")
    args = dict(args, r1=np.zeros_like(args["r1"]))
    with pytest.raises(api.PHFError):
        api.buildsc(*vec, args["nocc"], args["ngrid"], args["qj"], args["r1"], args["r2"], args["rpg"],
                    np.eye(M, dtype=complex)[None], args["roota"], args["rootb"], args["rooty"], args["weightsp"],
                    args["weightpg"], args["fsp"], args["fpg"], [1.0])
