"""F X = (H1 + J - K) X on the int8 path (phf_int8_fock_product).

Plans that form their densities with the int8 GEMM (int8 slices, n > 64) also form the per-point
product F_w X_w as one batched int8 GEMM over the chunk's points: X's columns and F's rows become
int8 slices (k = 2M, real and imaginary parts interleaved), and the epilogue writes the complex
result in place of the FP64 product.  Checked against the same plan with the FP64 product and against
the spatial Cholesky C oracle, for the stored exchange matrix and the streamed form, with several
sub-batches of points (a cap of 1 and 7 points) and with one.

Tolerance (relative to the largest element): int8 slices (S = 5) 1e-9, as for the other int8 forms.
"""
import numpy as np
import pytest

from oracle import phf_oracle as orc
from oracle import phf_oracle_c as corc
from phf_pcc_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu


def _akw(p):
    kw = p.grid_kwargs()
    return dict(ngrid=kw["ngrid"], nci=kw["nci"], cmplxconj=kw["CmplxConj"], ncisp=kw["ncisp"], nocc=p.N,
                r1=kw["R1"], r2=kw["R2"], rpg=kw["Rpg"], weightsp=kw["weightsp"], weightpg=kw["weightpg"],
                roota=kw["roota"], rootb=kw["rootb"], rooty=kw["rooty"], qj=kw["QJ"], sp=kw["SP"])


def _err(a, b):
    return float(np.abs(a - b).max()) / max(1.0, float(np.abs(b).max()))


class _fock(object):
    def __init__(self, on):
        self.on = on

    def __enter__(self):
        self.was = _lib.load().phf_int8_fock_product(self.on)

    def __exit__(self, *exc):
        _lib.load().phf_int8_fock_product(self.was)


def _run(p, Ref, Z, on, **kw):
    with _fock(on):
        with api.Plan(ref=Ref, h=p.h, B=p.B, precision="ozaki_i8", **_akw(p), **kw) as plan:
            return plan.buildhsg(Z, check_hermitian=False)


@pytest.mark.parametrize("n,N,L,jk,cap", [(65, 6, 40, "eri", 1), (96, 10, 50, "streamed", 7),
                                          (130, 20, 60, "streamed", 0)])
def test_int8_fock_product_matches_fp64_product_and_oracle(n, N, L, jk, cap):
    p = synth.make_problem(n, N, L, ngrid=(6, 3), seed=n, pg="C2v" if n < 128 else "None")
    Ref, Z = p.ref_and_z()
    Z = Z + 0.05 * np.random.default_rng(n).normal(size=Z.shape)
    kw = p.grid_kwargs()
    ora = corc.buildhsg(HOne=orc.mo_transform_1(p.hone_ao(), Ref), HTwo=None, Ref=Ref, Z=Z, Bs=p.B, **kw)
    fp64_fx = _run(p, Ref, Z, 0, jk_form=jk)
    int8_fx = _run(p, Ref, Z, cap if cap else 1, jk_form=jk)
    for x, y, z, key in zip(int8_fx, fp64_fx, ora, ("Hmat", "Smat", "Gradmat", "Rdmmat")):
        assert np.all(np.isfinite(x))
        assert _err(x, y) <= 1e-9, (key, _err(x, y))
        assert _err(x, z) <= 1e-9, (key, _err(x, z))
    e = lambda r: r[0][0, 0].real / abs(r[1][0, 0].real)
    assert abs(e(int8_fx) - e(fp64_fx)) <= 1e-9


def test_exact_gradient_with_int8_fock_product():
    """The exact (ket-side) gradient reads Gamma and W, which the int8 F X feeds: energy and gradient
    with the int8 product against the FP64 product (1e-9), and the gradient against central
    differences (h = 1e-5, to 1e-5 relative) along one seeded direction."""
    import torch

    from phf_pcc_b200.autograd import energy_and_gradient

    p = synth.make_problem(70, 7, 30, ngrid=(6, 3), seed=70, pg="C2v")
    C = torch.from_numpy(p.C).cuda()
    out = {}
    for on in (0, 1):
        with _fock(on):
            with api.Plan(ref=np.eye(p.M), h=p.h, B=p.B, precision="ozaki_i8", gradient="exact",
                          **_akw(p)) as plan:
                E, G = energy_and_gradient(C, plan)
                out[on] = (E.item(), G.clone())
                if on:
                    d = np.random.default_rng(5).normal(size=C.shape) + 1j * np.random.default_rng(6).normal(size=C.shape)
                    d = torch.from_numpy(d / np.linalg.norm(d)).cuda()
                    hstep = 1e-5
                    ep, _ = energy_and_gradient(C + hstep * d, plan)
                    em, _ = energy_and_gradient(C - hstep * d, plan)
                    fd = (ep - em).item() / (2 * hstep)
                    an = torch.real(torch.sum(torch.conj(2.0 * G) * d)).item()
                    # int8 energies carry ~1e-12 relative rounding that differences over 2h amplify; the
                    # bra-side-only gradient would be off by ~1e-3 on this coarse grid
                    assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (fd, an)
    assert abs(out[1][0] - out[0][0]) <= 1e-9 * max(1.0, abs(out[0][0]))
    gd = (out[1][1] - out[0][1]).abs().max().item()
    assert gd <= 1e-9 * max(1.0, out[0][1].abs().max().item()), gd


def test_fock_product_setting_round_trips():
    lib = _lib.load()
    was = lib.phf_int8_fock_product(0)
    try:
        assert lib.phf_int8_fock_product(1) == 0
        assert lib.phf_int8_fock_product(5) == 1
        assert lib.phf_int8_fock_product(1) == 5
    finally:
        lib.phf_int8_fock_product(was)
