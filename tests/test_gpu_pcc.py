"""The projected-CC grid kernel on the GPU (phf_pbarhbarolap through the C ABI, as PUCC_X2.fpucc) against
the oracle (oracle/phf_pcc.py, the numpy restatement of PbarHbarOlap / EvalKernel).

Cases: full spin projection (SP = 1) with and without C2v, J = 1 Wigner weights with random fsp / fpg,
Sz projection (SP = 2, ProjSz) on spin-blocked orbitals, the ncik = 2 pass (conjugated Hamiltonian and
amplitudes, Rk(2), fk(2)), grid points split over several chunks, and the configuration-1 size
(n = 20, M = 40, N = 10) on six grid points.  Tolerance: 1e-10 of the largest element of each output
(FP64 on both sides; the GPU sums the same terms in another order)."""
import numpy as np
import pytest

from oracle import phf_pcc as pcc
from phf_pcc_b200 import synth
from phf_pcc_b200.PUCC_X2 import fpucc

pytestmark = pytest.mark.gpu

NAMES = ("Olap0", "OlapEx1", "OlapEx2", "EOlap0", "EOlapEx1", "EOlapEx2")


def _problem(n, N, ngrid, seed, pg="None", SP=1, J=0, spin_blocked=False, ncik=1, rand_f=False):
    p = pcc.make_pcc_problem(n, N, 4 * n, ngrid=ngrid, seed=seed, pg=pg, SP=SP, J=J, spin_blocked=spin_blocked)
    p.pop("MO")
    rng = np.random.default_rng(seed + 11)
    cz = lambda *s: rng.normal(size=s) + 1j * rng.normal(size=s)
    if rand_f:
        p["fsp"] = cz(len(p["fsp"]))
        p["fpg"] = cz(len(p["fpg"]))
    if ncik == 2:
        M = p["HOne"].shape[0]
        p["ncik"] = 2
        p["Rk"] = np.array([np.eye(M), synth.random_unitary(M, rng)])
        p["fk"] = np.array([1.0, 0.7 - 0.4j])
    return p


def _gpu(p, workspace=0):
    M = p["HOne"].shape[0]
    o = p["NOcc"]
    args = (p["HOne"], p["HTwo"], None, p["T1"], p["T2"], o, M // 2, M, p["ENuc"], p["QJ"], p["SP"], p["NPoints"],
            p["Npg"], len(p["fsp"]), len(p["fpg"]), p["ncik"], p["R1"], p["R2"], p["Rpg"], p["Rk"], p["Roota"],
            p["Rootb"], p["Rooty"], p["Weightsp"], p["Weightpg"], p["fsp"], p["fpg"], p["fk"], p["TrunODE"])
    if workspace:
        from phf_pcc_b200 import api
        return api.pbarhbarolap(*args, workspace=workspace)
    return fpucc.pbarhbarolap(*args)


def _compare(got, ref, tol=1e-10):
    for name, g, r in zip(NAMES, got, ref):
        g, r = np.asarray(g), np.asarray(r)
        scale = max(np.abs(r).max(), 1e-300)
        err = np.abs(g - r).max() / scale
        assert err < tol, f"{name}: relative error {err:.3e}"


@pytest.mark.parametrize("case", [
    dict(n=4, N=4, ngrid=(6, 4), seed=1),
    dict(n=4, N=4, ngrid=(6, 2), seed=2, pg="C2v", J=1, rand_f=True),
    dict(n=4, N=4, ngrid=(1, 4), seed=3, SP=2, spin_blocked=True),
    dict(n=3, N=2, ngrid=(6, 2), seed=4, ncik=2),
    dict(n=5, N=4, ngrid=(6, 3), seed=5, pg="C2v"),
])
def test_pbarhbarolap_matches_oracle(case):
    p = _problem(**case)
    ref = pcc.pbarhbarolap(**p)
    got = _gpu(p)
    assert got[2].flags.f_contiguous and got[5].flags.f_contiguous
    _compare(got, ref)


@pytest.mark.parametrize("case", [
    dict(n=4, N=4, ngrid=(6, 2), seed=8),
    dict(n=5, N=4, ngrid=(6, 2), seed=9, pg="C2v", SP=1),
    dict(n=4, N=4, ngrid=(1, 3), seed=10, SP=2, spin_blocked=True),
])
def test_pbarhbarolap_with_triples_matches_oracle(case):
    """TrunODE 3: the (T) energy of the transformed amplitudes added to eps0 at every point (CCSD_T.f90);
    TrunODE -3 is the SD kernel (the reference adds (T) only for +3)."""
    p = _problem(**case)
    p["TrunODE"] = 3
    _compare(_gpu(p), pcc.pbarhbarolap(**p))
    p["TrunODE"] = -3
    _compare(_gpu(p), pcc.pbarhbarolap(**p))


def test_triples_split_over_sub_batches():
    """With (T): the default workspace runs the W-tensor GEMM path; a 64 KiB workspace (one grid point per
    chunk, no room for W) runs the fused shared-memory kernel.  Both give the oracle's sums."""
    p = _problem(6, 4, (6, 4), seed=12)
    p["TrunODE"] = 3
    whole = _gpu(p)
    _compare(whole, pcc.pbarhbarolap(**p))
    small = _gpu(p, workspace=1 << 16)
    _compare(small, whole, tol=1e-12)


def test_triples_tensor_path_large_occupied_space():
    """o = 20, above the fused (T) kernel's o <= 18: the W-tensor GEMM path at the configuration-1 size."""
    p = _problem(20, 20, (6, 1), seed=13)
    p["TrunODE"] = 3
    _compare(_gpu(p), pcc.pbarhbarolap(**p))


def test_chunked_grid_equals_one_chunk():
    p = _problem(4, 4, (6, 4), seed=6)
    whole = _gpu(p)
    small = _gpu(p, workspace=5 * 3 * (8 ** 4) * 16 * 4)  # a few points per chunk
    _compare(small, whole, tol=1e-12)


def test_configuration1_size_on_six_points():
    """n = 20 (M = 40), N = 10: the configuration-1 Hamiltonian generator with PCC amplitudes, on the six
    Lebedev points of a one-gamma grid."""
    p = _problem(20, 10, (6, 1), seed=7)
    ref = pcc.pbarhbarolap(**p)
    got = _gpu(p)
    _compare(got, ref)
    ene, _, r1, r2 = fpucc.pbarhbarresfromolap(None, *got, 10, 20, 40, 1)
    e_ref, _, r1_ref, r2_ref = pcc.pbarhbar_res_from_olap(*ref, 10, 40, 1)
    assert abs(ene - e_ref) < 1e-9 and np.abs(r1 - r1_ref).max() < 1e-9 and np.abs(r2 - r2_ref).max() < 1e-9
