"""The BuildSC oracle (oracle/phf_buildsc.py) on the properties of the reference's algorithm.

No reference output exists for BuildSC (Fortran behind a closed binary), so the restatement is held
to what PHF_fort/PHFTools.f90:464-537 and BuildSC_dr.f90 imply: the result is linear in the vector
(c0, c1, c2) (the overlap normalisation does not depend on it); with c1 = c2 = 0 it is
t0 = c0, t1 = c0 <Y>, t2 = c0 <Y_ac Y_bd - Y_ad Y_bc>, <.> the normalised projected average; and
for one grid point with R = I it is BuildSC_Vec of the untransformed vector with Y the occupied
projector.
"""
import numpy as np

from oracle.phf_buildsc import buildsc, buildsc_vec
from phf_pcc_b200 import synth


def _problem(n=3, N=2, seed=0, pg="C2v", J=0):
    p = synth.make_problem(n, N, 4, ngrid=(6, 3), seed=seed, pg=pg, J=J)
    g = p.grid
    rng = np.random.default_rng(seed)
    M = p.M
    cz = lambda *s: rng.normal(size=s) + 1j * rng.normal(size=s)
    fsp = cz(g.ncisp) if g.ncisp > 1 else np.ones(1, complex)
    fpg = cz(g.ncipg) if g.ncipg > 1 else np.ones(1, complex)
    U = p.Qfull  # rotations in an MO basis (as LinDep.py passes them), so the projection is generic
    mo = lambda R: np.einsum("ai,gab,bj->gij", U.conj(), R, U)
    args = dict(nocc=N, ngrid=g.ngrid, qj=g.J, r1=mo(g.R1), r2=mo(g.R2), rpg=mo(g.Rpg), roota=g.roota,
                rootb=g.rootb, rooty=g.rooty, weightsp=g.weightsp, weightpg=g.weightpg, fsp=fsp, fpg=fpg)
    vec = (complex(cz(1)[0]), 0.3 * cz(M, M), 0.1 * cz(M, M, M, M))
    return p, args, vec, cz


def test_buildsc_is_linear_in_the_vector():
    p, args, v, cz = _problem()
    M = p.M
    w = (complex(cz(1)[0]), 0.3 * cz(M, M), 0.1 * cz(M, M, M, M))
    a, b = 0.7 - 0.2j, -1.3 + 0.5j
    lin = tuple(a * x + b * y for x, y in zip(v, w))
    r = buildsc(*lin, **args)
    rv, rw = buildsc(*v, **args), buildsc(*w, **args)
    for x, y, z in zip(r, rv, rw):
        ref = a * np.asarray(y) + b * np.asarray(z)
        assert np.abs(np.asarray(x) - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_buildsc_scalar_channel():
    p, args, v, _ = _problem(seed=2)
    M = p.M
    c0 = 0.4 + 0.9j
    t0, t1, t2 = buildsc(c0, np.zeros((M, M)), np.zeros((M, M, M, M)), **args)
    assert abs(t0 - c0) <= 1e-13
    # t2 / c0 = <Y_ac Y_bd - Y_ad Y_bc> and t1 / c0 = <Y>: the same weights, so t2 follows from the
    # per-point densities; check the antisymmetry it must have
    assert np.abs(t2 + np.transpose(t2, (0, 1, 3, 2))).max() <= 1e-12 * np.abs(t2).max()
    assert np.abs(t2 + np.transpose(t2, (1, 0, 2, 3))).max() <= 1e-12 * np.abs(t2).max()


def test_buildsc_identity_point_is_buildsc_vec():
    p, args, v, _ = _problem(seed=3, pg="None")
    M, N = p.M, p.N
    one = dict(args, ngrid=(1, 1), r1=np.eye(M, dtype=complex)[None], r2=np.eye(M, dtype=complex)[None],
               rpg=np.eye(M, dtype=complex)[None], weightsp=np.ones((1, 1)), weightpg=np.ones((1, 1, 1)))
    Y = np.zeros((M, M), complex)
    Y[:N, :N] = np.eye(N)
    r = buildsc(*v, **one)
    ref = buildsc_vec(*v, Y)
    for x, y in zip(r, ref):
        assert np.abs(np.asarray(x) - np.asarray(y)).max() <= 1e-12 * max(1.0, np.abs(np.asarray(y)).max())
