"""Host-side API over the C ABI: one-shot calls and reusable plans.

All arrays follow the reference's conventions (complex128 spin-orbital matrices in
[alpha; beta] order, Fortran shapes of PHF_fort/PHFTools.f90:15-26).  The compute runs in
libphf_b200.so on the GPU; this module only converts and checks arguments.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PREC, PHFError, check, phf_complex, phf_plan_desc

__all__ = ["buildhsg", "buildhsg_chol", "localg", "buildsc", "pbarhbarolap", "Plan", "eval_batch", "check_status",
           "PHFError"]


def _fz(a):
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


def _fd(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


class _Grid:
    """Grid arguments of buildhsg converted to the C ABI layouts (kept alive by the instance)."""

    def __init__(self, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota, rootb, rooty,
                 qj, sp, npg=None, ncipg=None, nso=None):
        self.r1, self.r2, self.rpg = _fz(r1), _fz(r2), _fz(rpg)
        if self.r1.ndim != 3 or self.r2.ndim != 3 or self.rpg.ndim != 3:
            raise ValueError("r1, r2, rpg must be (count, nso, nso) arrays")
        self.nso = int(nso) if nso is not None else int(self.rpg.shape[1])
        self.npg = int(npg) if npg is not None else int(self.rpg.shape[0])
        self.weightpg = _fd(weightpg)
        self.ncipg = int(ncipg) if ncipg is not None else int(self.weightpg.shape[1])
        self.ngrid = np.ascontiguousarray(np.asarray(ngrid, dtype=np.int32).reshape(2))
        self.weightsp = _fd(weightsp)
        self.roota = np.ascontiguousarray(np.atleast_1d(np.asarray(roota, dtype=np.float64)))
        self.rootb = np.ascontiguousarray(np.atleast_1d(np.asarray(rootb, dtype=np.float64)))
        self.rooty = np.ascontiguousarray(np.atleast_1d(np.asarray(rooty, dtype=np.float64)))
        self.nci, self.cmplxconj, self.ncisp, self.nocc = int(nci), int(cmplxconj), int(ncisp), int(nocc)
        self.qj, self.sp = int(qj), int(sp)
        nl, ny = int(self.ngrid[0]), int(self.ngrid[1])
        M = self.nso
        if self.r1.shape != (nl, M, M) or self.r2.shape != (ny, M, M) or self.rpg.shape != (self.npg, M, M):
            raise ValueError(f"rotation shapes {self.r1.shape}, {self.r2.shape}, {self.rpg.shape} do not match "
                             f"ngrid={list(self.ngrid)}, npg={self.npg}, nso={M}")
        if self.weightsp.shape != (nl, ny):
            raise ValueError(f"weightsp shape {self.weightsp.shape} != {(nl, ny)}")
        if self.weightpg.shape != (self.npg, self.ncipg, self.ncipg):
            raise ValueError(f"weightpg shape {self.weightpg.shape} != {(self.npg, self.ncipg, self.ncipg)}")
        need_b = ny if self.sp == 2 else nl
        need_y = nl if self.sp == 2 else ny
        if self.roota.size < nl or self.rootb.size < need_b or self.rooty.size < need_y:
            raise ValueError("roota/rootb/rooty are shorter than the grid")

    def fill(self, d: phf_plan_desc):
        d.nso, d.nocc = self.nso, self.nocc
        d.ngrid = _ptr(self.ngrid)
        d.npg, d.nci, d.ncisp, d.ncipg = self.npg, self.nci, self.ncisp, self.ncipg
        d.cmplxconj, d.qj, d.sp = self.cmplxconj, self.qj, self.sp
        d.r1, d.r2, d.rpg = _ptr(self.r1), _ptr(self.r2), _ptr(self.rpg)
        d.weightsp, d.weightpg = _ptr(self.weightsp), _ptr(self.weightpg)
        d.roota, d.rootb, d.rooty = _ptr(self.roota), _ptr(self.rootb), _ptr(self.rooty)

    def outputs(self):
        nci, M = self.nci, self.nso
        return (np.zeros((nci, nci), dtype=np.complex128, order="F"),
                np.zeros((nci, nci), dtype=np.complex128, order="F"),
                np.zeros((nci, nci, M, M), dtype=np.complex128, order="F"),
                np.zeros((nci, nci, M, M), dtype=np.complex128, order="F"))


def _z_array(z, nso, nocc):
    z = _fz(z)
    if z.shape != (nso - nocc, nocc):
        raise ValueError(f"z shape {z.shape} != {(nso - nocc, nocc)}")
    return z


def _bvec_fortran(B, n):
    """Cholesky vectors B[L, p, q] (shape (L, n, n)) as the (n, n, L) Fortran array of the C ABI."""
    B = np.asarray(B, dtype=np.float64)
    if B.ndim != 3 or B.shape[1:] != (n, n):
        raise ValueError(f"Cholesky vectors must have shape (L, {n}, {n}), got {B.shape}")
    return np.asfortranarray(np.transpose(B, (1, 2, 0)))


def buildhsg(hone, htwo, ref, z, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota,
             rootb, rooty, qj, sp, npg=None, ncipg=None, nso=None, check_hermitian=True):
    """BuildHSG with a dense HTwo (PHF_fort/PHFTools.f90:10-201) on the GPU.

    Returns (Hmat, Smat, Gradmat, Rdmmat).  Raises PHFError where the reference STOPs; with
    ``check_hermitian=False`` a non-Hermitian result is returned instead."""
    g = _Grid(ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota, rootb, rooty, qj, sp,
              npg, ncipg, nso)
    M = g.nso
    hone, htwo, ref = _fz(hone), _fz(htwo), _fz(ref)
    if hone.shape != (M, M) or htwo.shape != (M, M, M, M) or ref.shape != (M, M):
        raise ValueError("hone/htwo/ref shapes do not match nso")
    z = _z_array(z, M, g.nocc)
    H, S, G, R = g.outputs()
    lib = _lib.load()
    st = lib.phf_buildhsg(_ptr(hone), _ptr(htwo), _ptr(ref), _ptr(z), _ptr(g.ngrid), g.npg, g.nci, g.cmplxconj,
                          g.ncisp, g.ncipg, g.nocc, M, _ptr(g.r1), _ptr(g.r2), _ptr(g.rpg), _ptr(g.weightsp),
                          _ptr(g.weightpg), _ptr(g.roota), _ptr(g.rootb), _ptr(g.rooty), g.qj, g.sp, _ptr(H),
                          _ptr(S), _ptr(G), _ptr(R))
    if st == _lib.PHF_ERR_NOT_HERMITIAN and not check_hermitian:
        return H, S, G, R
    check(st, "phf_buildhsg")
    return H, S, G, R


def buildhsg_chol(h, B, ref, z, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota, rootb,
                  rooty, qj, sp, npg=None, ncipg=None, nso=None, precision="fp64", check_hermitian=True):
    """BuildHSG with Cholesky two-electron integrals (see phf_buildhsg_chol in include/phf_b200.h)."""
    g = _Grid(ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota, rootb, rooty, qj, sp,
              npg, ncipg, nso)
    M = g.nso
    n = M // 2
    h = _fd(h)
    bvec = _bvec_fortran(B, n)
    ref = _fz(ref)
    z = _z_array(z, M, g.nocc)
    H, S, G, R = g.outputs()
    lib = _lib.load()
    st = lib.phf_buildhsg_chol(_ptr(h), _ptr(bvec), bvec.shape[2], _ptr(ref), _ptr(z), _ptr(g.ngrid), g.npg, g.nci,
                               g.cmplxconj, g.ncisp, g.ncipg, g.nocc, M, _ptr(g.r1), _ptr(g.r2), _ptr(g.rpg),
                               _ptr(g.weightsp), _ptr(g.weightpg), _ptr(g.roota), _ptr(g.rootb), _ptr(g.rooty), g.qj,
                               g.sp, PREC[precision], _ptr(H), _ptr(S), _ptr(G), _ptr(R))
    if st == _lib.PHF_ERR_NOT_HERMITIAN and not check_hermitian:
        return H, S, G, R
    check(st, "phf_buildhsg_chol")
    return H, S, G, R


def localg(gradmat, rdmmat, smat, e0, fsp, fpg, fk, cmplxconj, nso=None, nci=None, ncisp=None, ncipg=None):
    """LocalG (PHF_fort/PHFTools.f90:203-247) on the GPU; returns the full (nso, nso) G."""
    gradmat, rdmmat, smat = _fz(gradmat), _fz(rdmmat), _fz(smat)
    fsp = np.ascontiguousarray(np.atleast_1d(np.asarray(fsp, dtype=np.complex128)))
    fpg = np.ascontiguousarray(np.atleast_1d(np.asarray(fpg, dtype=np.complex128)))
    fk = np.ascontiguousarray(np.atleast_1d(np.asarray(fk, dtype=np.complex128)))
    nci = int(nci) if nci is not None else gradmat.shape[0]
    nso = int(nso) if nso is not None else gradmat.shape[2]
    ncisp = int(ncisp) if ncisp is not None else fsp.size
    ncipg = int(ncipg) if ncipg is not None else fpg.size
    if int(cmplxconj) == 2 and fk.size < 2:
        raise ValueError("fk needs 2 entries when cmplxconj == 2")
    G = np.zeros((nso, nso), dtype=np.complex128, order="F")
    e = complex(np.asarray(e0).item())
    lib = _lib.load()
    st = lib.phf_localg(_ptr(gradmat), _ptr(rdmmat), _ptr(smat), phf_complex(e.real, e.imag), nso, _ptr(fsp),
                        _ptr(fpg), _ptr(fk), nci, ncisp, ncipg, int(cmplxconj), _ptr(G))
    check(st, "phf_localg")
    return G


def buildsc(c0, c1, c2, nocc, ngrid, qj, r1, r2, rpg, rk, roota, rootb, rooty, weightsp, weightpg, fsp, fpg, fk,
            nso=None, npg=None, ncisp=None, ncipg=None, ncik=None):
    """BuildSC (PHF_fort/PHFTools.f90:464-537) on the GPU: (t0, t1 (M, M), t2 (M, M, M, M)) for the vector
    (c0, c1, c2), Fortran-ordered complex128 outputs (see phf_buildsc in include/phf_b200.h)."""
    c1, c2 = _fz(c1), _fz(c2)
    M = int(nso) if nso is not None else c1.shape[0]
    if c1.shape != (M, M) or c2.shape != (M, M, M, M):
        raise ValueError("c1 must be (M, M) and c2 (M, M, M, M)")
    r1, r2, rpg, rk = _fz(r1), _fz(r2), _fz(rpg), _fz(rk)
    ng = np.ascontiguousarray(np.asarray(ngrid, dtype=np.int32).reshape(2))
    npg = int(npg) if npg is not None else rpg.shape[0]
    wsp, wpg = _fd(weightsp), _fd(weightpg)
    fsp_, fpg_, fk_ = (np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.complex128))) for x in (fsp, fpg, fk))
    ncisp = int(ncisp) if ncisp is not None else fsp_.size
    ncipg = int(ncipg) if ncipg is not None else fpg_.size
    ncik = int(ncik) if ncik is not None else fk_.size
    if r1.shape != (int(ng[0]), M, M) or r2.shape != (int(ng[1]), M, M) or rpg.shape != (npg, M, M):
        raise ValueError("rotation shapes do not match ngrid, npg and nso")
    ra, rb, ry = (np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float64))) for x in (roota, rootb, rooty))
    c0c = complex(np.asarray(c0).item())
    t0 = phf_complex()
    t1 = np.zeros((M, M), dtype=np.complex128, order="F")
    t2 = np.zeros((M, M, M, M), dtype=np.complex128, order="F")
    st = _lib.load().phf_buildsc(phf_complex(c0c.real, c0c.imag), _ptr(c1), _ptr(c2), int(nocc), M, _ptr(ng), npg,
                                 int(qj), ncisp, ncipg, ncik, _ptr(r1), _ptr(r2), _ptr(rpg), _ptr(rk), _ptr(ra),
                                 _ptr(rb), _ptr(ry), _ptr(wsp), _ptr(wpg), _ptr(fsp_), _ptr(fpg_), _ptr(fk_),
                                 ctypes.byref(t0), _ptr(t1), _ptr(t2))
    check(st, "phf_buildsc")
    return complex(t0.re, t0.im), t1, t2


def pbarhbarolap(hone, htwo, ref, t1, t2, nocc, nao, nso, enuc, qj, sp, npoints, npg, ncisp, ncipg, ncik, r1, r2,
                 rpg, rk, roota, rootb, rooty, weightsp, weightpg, fsp, fpg, fk, trunode, comm=None, workspace=0):
    """PbarHbarOlap (SUCCSD_Boson_cmplx/FPUCC.f90:14-272), the projected-CCSD grid kernel, on the GPU.

    Arguments in the order of the Fortran dummy arguments after the outputs; returns
    (Olap0, OlapEx1 (v, nocc), OlapEx2 (v, v, nocc, nocc), EOlap0, EOlapEx1, EOlapEx2) as complex scalars
    and Fortran-ordered complex128 arrays (v = nso - nocc).  ``ref`` and ``nao`` are accepted and not used,
    as in the reference; ``comm`` is not used (the grid is not split over ranks here).  ``workspace``:
    device bytes per chunk of grid points (0 = 16 GiB).  See phf_pbarhbarolap in include/phf_b200.h."""
    del comm
    M, o = int(nso), int(nocc)
    v = M - o
    hone_, htwo_, t1_, t2_ = _fz(hone), _fz(htwo), _fz(t1), _fz(t2)
    if hone_.shape != (M, M) or htwo_.shape != (M, M, M, M) or t1_.shape != (v, o) or t2_.shape != (v, v, o, o):
        raise ValueError("hone (M, M), htwo (M, M, M, M), t1 (v, o) and t2 (v, v, o, o) expected")
    ng = np.ascontiguousarray(np.asarray(npoints, dtype=np.int32).reshape(2))
    r1_, r2_, rpg_, rk_ = _fz(r1), _fz(r2), _fz(rpg), _fz(rk)
    if r1_.shape != (int(ng[0]), M, M) or r2_.shape != (int(ng[1]), M, M) or rpg_.shape != (int(npg), M, M):
        raise ValueError("rotation shapes do not match npoints, npg and nso")
    if rk_.ndim != 3 or rk_.shape[0] < int(ncik) or rk_.shape[1:] != (M, M):
        raise ValueError("rk must be (ncik, nso, nso)")
    ra, rb, ry = (np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float64))) for x in (roota, rootb, rooty))
    wsp, wpg = _fd(weightsp), _fd(weightpg)
    fsp_, fpg_, fk_ = (np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.complex128))) for x in (fsp, fpg, fk))
    ref_ = _fz(ref) if ref is not None else None
    out0, oute0 = phf_complex(), phf_complex()
    ex1, eex1 = (np.zeros((v, o), dtype=np.complex128, order="F") for _ in range(2))
    ex2, eex2 = (np.zeros((v, v, o, o), dtype=np.complex128, order="F") for _ in range(2))
    st = _lib.load().phf_pbarhbarolap(
        ctypes.byref(out0), _ptr(ex1), _ptr(ex2), ctypes.byref(oute0), _ptr(eex1), _ptr(eex2), _ptr(hone_),
        _ptr(htwo_), _ptr(ref_), _ptr(t1_), _ptr(t2_), o, int(nao), M, float(enuc), int(qj), int(sp), _ptr(ng),
        int(npg), int(ncisp), int(ncipg), int(ncik), _ptr(r1_), _ptr(r2_), _ptr(rpg_), _ptr(rk_), _ptr(ra), _ptr(rb),
        _ptr(ry), _ptr(wsp), _ptr(wpg), _ptr(fsp_), _ptr(fpg_), _ptr(fk_), int(trunode), int(workspace))
    check(st, "phf_pbarhbarolap")
    return complex(out0.re, out0.im), ex1, ex2, complex(oute0.re, oute0.im), eex1, eex2


class Plan:
    """A reusable evaluation plan (Hamiltonian, grid and workspace resident on the GPU).

    Cholesky form: pass ``h`` (n, n) and ``B`` (L, n, n); dense form: ``hone`` and
    ``htwo``.  Grid arguments as buildhsg.  ``precision`` of the J/K contractions: "fp64",
    "ozaki_i8" (FP64-accurate int8 tensor-core slices, ``slices`` per operand, default 5),
    "bf16x3" (split BF16, three products) or "tf32" (both FP32-accumulated in 512-element segments
    summed in FP64; about 1e-6 relative, far from FP64); ``jk_form``: "auto", "eri"
    (exchange through the n^2 x n^2 spatial ERI matrix, built once and kept), "streamed" (the same
    exchange rows regenerated from the Cholesky vectors panel by panel in every chunk: no n^4
    tensor, ``exchange_panel`` spatial indices per panel, 0 = automatic) or "factorized" (rank-N
    J/K, FP64 only); "auto" takes "eri" up to n = 128 and "streamed" above.  ``gradient``:
    "reference" (the reference's bra-side gradient, LocalG) or "exact" (dE/dC* including the
    ket-side term; used by autograd).  ``autotune``: time the launch choices of the plan's GEMM shapes
    at its first evaluation (bitwise the same results).  ``exchange_symmetry`` (streamed form):
    "auto" (on where available), True or False -- with it the exchange runs over index pairs i <= k
    against the symmetric half of each density and i < k against the antisymmetric half (K(rho^T) =
    K(rho)^T for real integrals): half the exchange GEMM's work.  Available in FP64 and, for n > 64,
    in the tensor-core precisions."""

    def __init__(self, *, ref, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota, rootb,
                 rooty, qj, sp, h=None, B=None, hone=None, htwo=None, precision="fp64", slices=0,
                 workspace_bytes=0, jk_form="auto", gradient="reference", fp64_library_gemm=False,
                 point_range=None, npg=None, ncipg=None, nso=None, exchange_panel=0, autotune=False,
                 exchange_symmetry="auto"):
        self._g = _Grid(ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg, roota, rootb, rooty, qj,
                        sp, npg, ncipg, nso)
        g = self._g
        M = g.nso
        d = phf_plan_desc()
        g.fill(d)
        self._keep = []
        self.ref = _fz(ref)
        d.ref = _ptr(self.ref)
        if B is not None:
            self._h = _fd(h)
            self._b = _bvec_fortran(B, M // 2)
            d.nchol = self._b.shape[2]
            d.h, d.bvec = _ptr(self._h), _ptr(self._b)
        else:
            self._hone, self._htwo = _fz(hone), _fz(htwo)
            d.nchol = 0
            d.hone, d.htwo = _ptr(self._hone), _ptr(self._htwo)
        d.precision = PREC[precision]
        d.slices = int(slices)
        d.workspace_bytes = int(workspace_bytes)
        d.jk_form = {"auto": 0, "eri": 1, "factorized": 2, "streamed": 3}[jk_form]
        d.exchange_panel = int(exchange_panel)
        d.autotune = 1 if autotune else 0
        if exchange_symmetry == "auto" or exchange_symmetry is None:
            d.exchange_symmetry = 0
        else:
            d.exchange_symmetry = 1 if exchange_symmetry else 2
        self.jk_form = jk_form
        d.gradient_mode = {"reference": 0, "exact": 1}[gradient]
        d.fp64_library_gemm = 1 if fp64_library_gemm else 0
        if point_range is not None:
            d.point_begin, d.point_end = int(point_range[0]), int(point_range[1])
        self.gradient = gradient
        self.precision = precision
        handle = ctypes.c_void_p()
        lib = _lib.load()
        check(lib.phf_plan_create(ctypes.byref(d), ctypes.byref(handle)), "phf_plan_create")
        self._handle = handle
        # the Hamiltonian now lives on the device; drop the host copies
        self._h = self._b = self._hone = self._htwo = None
        self.nso, self.nocc, self.nci = M, g.nocc, g.nci

    @property
    def chunk(self) -> int:
        c = ctypes.c_int()
        s = ctypes.c_size_t()
        _lib.load().phf_plan_info(self._handle, ctypes.byref(c), ctypes.byref(s))
        return int(c.value)

    @property
    def workspace_bytes(self) -> int:
        c = ctypes.c_int()
        s = ctypes.c_size_t()
        _lib.load().phf_plan_info(self._handle, ctypes.byref(c), ctypes.byref(s))
        return int(s.value)

    def buildhsg(self, z, check_hermitian=True):
        z = _z_array(z, self.nso, self.nocc)
        H, S, G, R = self._g.outputs()
        st = _lib.load().phf_plan_buildhsg(self._handle, _ptr(z), _ptr(H), _ptr(S), _ptr(G), _ptr(R))
        if st == _lib.PHF_ERR_NOT_HERMITIAN and not check_hermitian:
            return H, S, G, R
        check(st, "phf_plan_buildhsg")
        return H, S, G, R

    def eval_device(self, C, out=None, stream=None):
        """Accumulators for a device-resident C (torch complex128 (M, N) CUDA tensor).

        Returns (hs (nci*nci, 2), yg (nci*nci, M, N), yr (nci*nci, M, N)) as torch tensors."""
        import torch

        if C.dtype != torch.complex128 or not C.is_cuda or tuple(C.shape) != (self.nso, self.nocc):
            raise ValueError(f"C must be a complex128 CUDA tensor of shape {(self.nso, self.nocc)}")
        C = C.contiguous()
        ns = self.nci * self.nci
        if out is None:
            hs = torch.empty((ns, 2), dtype=torch.complex128, device=C.device)
            yg = torch.empty((ns, self.nso, self.nocc), dtype=torch.complex128, device=C.device)
            yr = torch.empty_like(yg)
        else:
            hs, yg, yr = out
        if stream is None:
            stream = torch.cuda.current_stream(C.device)
        st = _lib.load().phf_plan_eval_device(self._handle, ctypes.c_void_p(C.data_ptr()),
                                              ctypes.c_void_p(hs.data_ptr()), ctypes.c_void_p(yg.data_ptr()),
                                              ctypes.c_void_p(yr.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        check(st, "phf_plan_eval_device")
        return hs, yg, yr

    def eval_device_async(self, C, out, status, stream=None):
        """eval_device without the host synchronisation (phf_plan_eval_device_async): queues the
        evaluation on ``stream`` and returns at once; ``out`` = (hs, yg, yr) as eval_device returns
        them and ``status`` an int32 CUDA tensor of 2 that receives the status words (see
        ``check_status``) on the same stream."""
        import torch

        if C.dtype != torch.complex128 or not C.is_cuda or tuple(C.shape) != (self.nso, self.nocc) or \
                not C.is_contiguous():
            raise ValueError(f"C must be a contiguous complex128 CUDA tensor of shape {(self.nso, self.nocc)}")
        if status.dtype != torch.int32 or not status.is_cuda or status.numel() < 2:
            raise ValueError("status must be an int32 CUDA tensor of at least 2 elements")
        hs, yg, yr = out
        if stream is None:
            stream = torch.cuda.current_stream(C.device)
        st = _lib.load().phf_plan_eval_device_async(
            self._handle, ctypes.c_void_p(C.data_ptr()), ctypes.c_void_p(hs.data_ptr()),
            ctypes.c_void_p(yg.data_ptr()), ctypes.c_void_p(yr.data_ptr()), ctypes.c_void_p(status.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream))
        check(st, "phf_plan_eval_device_async")
        return hs, yg, yr

    def close(self):
        if getattr(self, "_handle", None):
            _lib.load().phf_plan_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def check_status(words):
    """Raise PHFError for the status words of phf_plan_eval_device_async (host ints)."""
    flag, oz = int(words[0]), int(words[1])
    if oz:
        raise PHFError(_lib.PHF_ERR_CUDA, f"tensor-core GEMM pipeline wait timed out (code {oz})")
    if flag & 1:
        raise PHFError(_lib.PHF_ERR_SINGULAR, "a rotated overlap bra^H R ket is exactly singular")
    if flag & 2:
        raise PHFError(_lib.PHF_ERR_NONFINITE, "non-finite rotated overlap")


def eval_batch(plans, Cs, outs=None, stream=None):
    """Evaluate independent instances together (phf_eval_batch): plans[i] at the device-resident
    determinant Cs[i] (complex128 (M_i, N_i) CUDA tensors).  Returns one (hs, yg, yr) triple per
    instance, as Plan.eval_device.  All instances run as one CUDA graph, captured on the first call
    for this set of plans and buffers; pass the returned triples back as ``outs`` (and keep the same
    Cs tensors) to replay it without recapturing."""
    import torch

    if len(plans) != len(Cs):
        raise ValueError("one determinant per plan")
    if outs is None:
        outs = []
        for pl, C in zip(plans, Cs):
            ns = pl.nci * pl.nci
            yg = torch.empty((ns, pl.nso, pl.nocc), dtype=torch.complex128, device=C.device)
            outs.append((torch.empty((ns, 2), dtype=torch.complex128, device=C.device), yg, torch.empty_like(yg)))
    for pl, C in zip(plans, Cs):
        if C.dtype != torch.complex128 or not C.is_cuda or tuple(C.shape) != (pl.nso, pl.nocc) or \
                not C.is_contiguous():
            raise ValueError(f"each C must be a contiguous complex128 CUDA tensor of its plan's shape")
    n = len(plans)
    P = ctypes.c_void_p * n
    ptrs = lambda ts: P(*[ctypes.c_void_p(t.data_ptr()) for t in ts])
    if stream is None:
        stream = torch.cuda.current_stream(Cs[0].device if n else None)
    st = _lib.load().phf_eval_batch(P(*[pl._handle for pl in plans]), n, ptrs(Cs), ptrs([o[0] for o in outs]),
                                    ptrs([o[1] for o in outs]), ptrs([o[2] for o in outs]),
                                    ctypes.c_void_p(stream.cuda_stream))
    check(st, "phf_eval_batch")
    return outs
