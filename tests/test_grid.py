"""Projection-grid set-up against the reference's own RootWeight/RootWeightSy/BuildRotMat/WignerMat."""
import numpy as np
import pytest

from phf_pcc_b200 import grid
from tests._golden import load

G = load("grids")


@pytest.mark.parametrize("ng", [(6, 4), (14, 8), (26, 3), (38, 2), (50, 16)])
def test_root_weight_matches_reference(ng):
    key = f"rw_{ng[0]}_{ng[1]}"
    a, b, y, w = grid.root_weight(ng)
    ra, rb = G[key + "_a"], G[key + "_b"]
    # Lebedev points as sets (the orbit enumeration order may differ); weights by point
    mine = {(round(x, 9), round(z, 9)): wi for x, z, wi in zip(a, b, w[:, 0])}
    ref = {(round(x, 9), round(z, 9)): wi for x, z, wi in zip(ra, rb, G[key + "_w"][:, 0])}
    assert mine.keys() == ref.keys()
    for k in ref:
        assert abs(mine[k] - ref[k]) < 1e-14
    assert np.allclose(y, G[key + "_y"], atol=1e-15)
    assert abs(w.sum() - G[key + "_w"].sum()) < 1e-13


@pytest.mark.parametrize("ny", [1, 4, 7])
def test_root_weight_sy_matches_reference(ny):
    b, w = grid.root_weight_sy(ny)
    order = np.argsort(b)
    ro = np.argsort(G[f"sy_{ny}_b"])
    assert np.allclose(b[order], G[f"sy_{ny}_b"][ro], atol=1e-13)
    assert np.allclose(w[order], G[f"sy_{ny}_w"][ro], atol=1e-13)


def test_build_rot_mat_matches_reference():
    for args, R in zip(G["rot_args"], G["rot"]):
        assert np.allclose(grid.build_rot_mat(*args, 3), R, atol=1e-15)


def test_wigner_matches_reference():
    for args, v in zip(G["wig_args"], G["wig_vals"]):
        j, n, m = (int(round(x)) for x in args[:3])
        assert abs(grid.wigner_D(j, n, m, *args[3:]) - v) < 1e-13


def test_weights_sum_to_two_pi():
    for ng in [(14, 8), (50, 16)]:
        _, _, _, w = grid.root_weight(ng)
        assert abs(w.sum() - 2 * np.pi) < 1e-12


def test_spin_rotation_is_unitary_and_wigner_identity():
    for (a, b, y) in [(0.1, 0.2, 0.3), (2.0, 3.0, -1.0)]:
        U = grid.spin_rotation_2x2(a, b, y)
        assert np.allclose(U.conj().T @ U, np.eye(2))
        assert grid.wigner_D(0, 0, 0, a, b, y) == 1.0


def test_c2v_projector_characters():
    n = 7
    for irrep, ch in [("A1", (1, 1, 1, 1)), ("B1", (1, -1, 1, -1))]:
        ncipg, wpg, Rpg = grid.c2v_projector(n, irrep)
        assert ncipg == 1 and wpg.shape == (4, 1, 1)
        assert tuple(wpg[:, 0, 0]) == ch
        # group closure: C2 * sigma_xz = sigma_yz, each op squares to identity
        assert np.allclose(Rpg[1] @ Rpg[2], Rpg[3])
        for g in Rpg:
            assert np.allclose(g @ g, np.eye(2 * n))


@pytest.mark.parametrize("name", ["e_c4v", "j1_e_c4v"])
def test_c4v_projector_matches_reference_table(name):
    """grid.c4v_projector's E-irrep weights and operations against the golden cases, whose weights
    came from the reference's own C4vTable (PGSymm.py:109-137)."""
    c = load(name)
    ncipg, w, R = grid.c4v_projector(int(c["n"]), "E")
    assert ncipg == int(c["ncipg"]) == 2
    assert np.array_equal(w, c["weightpg"])
    assert np.array_equal(R, c["Rpg"])
    # a representation: the orbital operations multiply like the E matrices (C4 C4 = C2, C4 sigma_xz = sigma_d)
    ops = grid.c4v_orbital_ops(int(c["n"]))
    E = grid.c4v_e_matrices()
    for a, b, ab in ((1, 1, 2), (1, 4, 6), (2, 4, 5), (3, 4, 7)):
        assert np.allclose(ops[a] @ ops[b], ops[ab]) and np.allclose(E[a] @ E[b], E[ab])
