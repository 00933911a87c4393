"""The differentiable projected energy: values against the golden vectors, gradient against
central finite differences (h = 1e-5) and against the reference's own gradient (LocalG)."""
import numpy as np
import pytest

from phf_pcc_b200 import api, synth
from phf_pcc_b200.autograd import energy_and_gradient, projected_energy
from tests._golden import grid_kwargs, load

pytestmark = pytest.mark.gpu


def _plan_kwargs_from_grid(kw, nocc):
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=nocc,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


@pytest.mark.parametrize("precision", ["fp64", "ozaki_i8"])
def test_energy_and_gradient_match_reference_golden(precision):
    import torch

    c = load("c1")
    M, N = int(c["M"]), int(c["N"])
    C = c["Ref"] @ np.vstack([np.eye(N), c["Z"]])
    with api.Plan(ref=np.eye(M), h=c["h"], B=c["B"], precision=precision,
                  **_plan_kwargs_from_grid(grid_kwargs(c), N)) as plan:
        Ct = torch.from_numpy(C).cuda().requires_grad_(True)
        E = projected_energy(Ct, plan)
        E.backward()
        g = Ct.grad.cpu().numpy() / 2.0          # dE/dC*
    assert abs(E.item() - c["E0"]) <= 1e-9
    Gz = (c["Ref"].conj().T @ g)[N:, :]           # dE/dZ* in the Ref-MO basis
    assert np.abs(Gz - c["G"]).max() <= 1e-8


@pytest.mark.parametrize("precision", ["fp64", "ozaki_i8"])
def test_gradient_matches_central_finite_differences(precision):
    """Exact-gradient plans against central differences on a coarse grid (14 x 8 x C2v) where the
    reference's bra-side gradient differs from dE/dC* at the 1e-3 level."""
    import torch

    p = synth.make_problem(16, 8, 40, ngrid=(14, 8), seed=21, pg="C2v")
    with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision=precision, gradient="exact",
                  **_plan_kwargs_from_grid(p.grid_kwargs(), p.N)) as plan:
        C = torch.from_numpy(p.C).cuda()
        E0, G = energy_and_gradient(C, plan)
        grad = 2.0 * G
        rng = np.random.default_rng(3)
        for _ in range(3):
            d = rng.normal(size=C.shape) + 1j * rng.normal(size=C.shape)
            d = torch.from_numpy(d / np.linalg.norm(d)).cuda()
            h = 1e-5
            ep, _ = energy_and_gradient(C + h * d, plan)
            em, _ = energy_and_gradient(C - h * d, plan)
            fd = (ep - em).item() / (2 * h)
            an = torch.real(torch.sum(torch.conj(grad) * d)).item()
            assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)


def test_exact_and_reference_gradients_agree_on_fine_symmetric_grid():
    """On the golden config-1 problem (grid 14 x 8, H/S real to 1e-16) both gradients coincide
    with the reference's LocalG."""
    import torch

    c = load("c1")
    M, N = int(c["M"]), int(c["N"])
    C = torch.from_numpy(c["Ref"] @ np.vstack([np.eye(N), c["Z"]])).cuda()
    out = {}
    for mode in ("reference", "exact"):
        with api.Plan(ref=np.eye(M), h=c["h"], B=c["B"], gradient=mode,
                      **_plan_kwargs_from_grid(grid_kwargs(c), N)) as plan:
            out[mode] = energy_and_gradient(C, plan)
    assert abs(out["exact"][0].item() - out["reference"][0].item()) < 1e-12
    diff = (out["exact"][1] - out["reference"][1]).abs().max().item()
    assert diff <= 1e-6 * out["reference"][1].abs().max().item(), diff


def test_config2_adjoint_twenty_rotation_steps_against_fd_and_reference_gradient():
    """Configuration-2 adjoint protocol (n = 64, M = 128, N = 32, L = 400, 50 x 16 x 4 C2v grid, int8
    slices): 20 seeded orbital-rotation steps C <- exp(kappa) C (anti-Hermitian kappa, N(0, 1e-2)).
    At each step the autograd gradient (exact-gradient plan, forward + backward) is checked

    * against central finite differences (h = 1e-5) along a random direction, to 1e-5 relative (the
      int8 energies carry ~1e-11 Eh of rounding, which the difference quotient divides by 2h: up to
      2.3e-6 relative was seen over the 20 steps);
    * against the reference's gradient: with Ref = I and the determinant in Thouless form
      [I; Z] = C C_occ^-1, LocalG's G[N:, :N] = dE/dZ* (PHF_fort/PHFTools.f90:203-247) from the
      reference-mode plan on the full grid equals the autograd gradient carried to Z by the chain
      rule (the bra-side and exact gradients differ only by the grid's Hermiticity defect), to 1e-5
      of max|G|;
    * and that reference gradient against the C oracle on a block of 4 grid points (the beta = 0
      Lebedev point): the block's LocalG gradient from the GPU plan and from the oracle within 1e-7,
      the block's energy within 1e-8 Eh."""
    import torch

    from oracle import phf_oracle_c as corc

    p = synth.config_problem("c2", seed=2)
    M, N = p.M, p.N
    kw = p.grid_kwargs()
    akw = _plan_kwargs_from_grid(kw, N)
    g = p.grid
    w0 = int(np.argmin(np.abs(np.asarray(g.rootb)))) * g.ngrid[1] * g.npg
    block = (w0, w0 + 4)
    rng = np.random.default_rng(11)

    def block_e_g(H, S, Gm, Rm):
        e = H[0, 0].real / abs(S[0, 0].real)
        G = api.localg(Gm, Rm, S, e, [1.0 / np.sqrt(abs(S[0, 0].real))], [1.0], [1.0], 1)
        return e, G[N:, :N]

    with api.Plan(ref=np.eye(M), h=p.h, B=p.B, precision="ozaki_i8", gradient="exact", **akw) as pe, \
            api.Plan(ref=np.eye(M), h=p.h, B=p.B, precision="ozaki_i8", **akw) as pr, \
            api.Plan(ref=np.eye(M), h=p.h, B=p.B, precision="ozaki_i8", point_range=block, **akw) as pb:
        C0 = p.C
        for step in range(20):
            C0 = synth.orbital_rotation(C0, 1e-2, rng)
            C = torch.from_numpy(C0).cuda().requires_grad_(True)
            E = projected_energy(C, pe)
            E.backward()
            grad = C.grad
            d = rng.normal(size=C0.shape) + 1j * rng.normal(size=C0.shape)
            d = torch.from_numpy(d / np.linalg.norm(d)).cuda()
            h = 1e-5
            with torch.no_grad():
                ep = projected_energy(C.detach() + h * d, pe)
                em = projected_energy(C.detach() - h * d, pe)
            fd = (ep - em).item() / (2 * h)
            an = torch.real(torch.sum(torch.conj(grad) * d)).item()
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (step, fd, an)
            # the reference's gradient on the full grid (bra side, LocalG), dE/dZ* at the Thouless form
            # [I; Z] = C0 A^-1 (A = C0[:N]) of the same determinant; E(C0) = E([I; Z] A), so
            # dE/dZ* = (dE/dC0* A^H)[N:, :]
            A = C0[:N]
            Z = C0[N:] @ np.linalg.inv(A)
            H, S, Gm, Rm = pr.buildhsg(Z, check_hermitian=False)
            e_ref, G_ref = block_e_g(H, S, Gm, Rm)
            gz = ((grad.cpu().numpy() / 2.0) @ A.conj().T)[N:, :]
            assert abs(e_ref - E.item()) <= 1e-9 * abs(E.item()), (step, e_ref, E.item())
            assert np.abs(gz - G_ref).max() <= 1e-5 * np.abs(G_ref).max(), (step, np.abs(gz - G_ref).max())
            # that gradient's machinery against the oracle on a block of grid points
            eb, gb = block_e_g(*pb.buildhsg(Z, check_hermitian=False))
            ora = corc.buildhsg(p.hone_ao(), None, np.eye(M), Z, Bs=p.B, omega_list=np.arange(*block), **kw)
            eo, go = block_e_g(*ora)
            assert abs(eb - eo) <= 1e-8, (step, eb, eo)
            assert np.abs(gb - go).max() <= 1e-7, (step, np.abs(gb - go).max())


def test_recompute_mode_equals_fused_mode():
    import torch

    p = synth.make_problem(12, 6, 30, ngrid=(14, 4), seed=4)
    with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, **_plan_kwargs_from_grid(p.grid_kwargs(), p.N)) as plan:
        grads = []
        for mode in ("fused", "recompute"):
            C = torch.from_numpy(p.C).cuda().requires_grad_(True)
            projected_energy(C, plan, mode).backward()
            grads.append(C.grad.clone())
    assert torch.equal(grads[0], grads[1])


def test_energy_invariant_under_occupied_rotation_at_config2_size():
    """Size-independent property at the benchmark size: E(C U) = E(C) for unitary U (N x N)."""
    import torch

    p = synth.config_problem("c2", seed=7)
    with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision="ozaki_i8",
                  **_plan_kwargs_from_grid(p.grid_kwargs(), p.N)) as plan:
        C = torch.from_numpy(p.C).cuda()
        U = torch.from_numpy(synth.random_unitary(p.N, np.random.default_rng(1))).cuda()
        E1, G1 = energy_and_gradient(C, plan)
        E2, G2 = energy_and_gradient(C @ U, plan)
    assert abs(E1.item() - E2.item()) <= 1e-9 * abs(E1.item())
    # the gradient transforms covariantly: G(C U) = G(C) U
    assert torch.allclose(G2, G1 @ U, rtol=0, atol=1e-9 * float(G1.abs().max()))
