"""ctypes wrapper of the C oracle (oracle/libphf_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/ as a faster FP64 checker and by bench.py as the timed CPU baseline
(a C restatement of PHF_fort/PHFTools.f90 BuildHSG/LocalG; see phf_oracle.c).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphf_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-C", HERE], stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_buildhsg.restype = ctypes.c_int
        _lib.oracle_buildhsg_ex.restype = ctypes.c_int
        _lib.oracle_localg.restype = ctypes.c_int
        _lib.oracle_num_threads.restype = ctypes.c_int
    return _lib


def _f(a, dtype=np.complex128):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def buildhsg(HOne, HTwo, Ref, Z, ngrid, nci, CmplxConj, ncisp, NOcc, R1, R2, Rpg, weightsp, weightpg,
             roota, rootb, rooty, QJ, SP, npg, ncipg, NSO, Bt=None, Bs=None, omega_list=None, nthreads=0):
    """Same contract as oracle.phf_oracle.buildhsg.  ``Bt`` (M, M, L) are MO-basis Cholesky
    vectors used instead of HTwo when HTwo is None; ``Bs`` (L, n, n) are the real spatial
    Cholesky vectors in the AO basis (the MO basis is Ref), used instead of both.  ``omega_list``:
    flattened grid-point indices ((il*ny + iy)*npg + ipg) to restrict the sum.  With fewer
    points than threads each point's work is split over the threads."""
    M = NSO
    keep = []
    hone = _f(HOne)
    htwo = _f(HTwo) if HTwo is not None else None
    bt = _f(Bt) if Bt is not None else None
    bs = _f(np.transpose(Bs, (1, 2, 0)), np.float64) if Bs is not None else None
    nchol = Bt.shape[2] if Bt is not None else (Bs.shape[0] if Bs is not None else 0)
    ref, z = _f(Ref), _f(Z)
    r1, r2, rpg = _f(R1), _f(R2), _f(Rpg)
    wsp, wpg = _f(weightsp, np.float64), _f(weightpg, np.float64)
    ra, rb, ry = (np.ascontiguousarray(x, dtype=np.float64) for x in (roota, rootb, rooty))
    ng = np.asarray(ngrid, dtype=np.int32)
    ol = None if omega_list is None else np.ascontiguousarray(omega_list, dtype=np.int32)
    hmat = np.zeros((nci, nci), dtype=np.complex128, order="F")
    smat = np.zeros((nci, nci), dtype=np.complex128, order="F")
    gmat = np.zeros((nci, nci, M, M), dtype=np.complex128, order="F")
    rmat = np.zeros((nci, nci, M, M), dtype=np.complex128, order="F")
    keep += [hone, htwo, bt, bs, ref, z, r1, r2, rpg, wsp, wpg, ra, rb, ry, ng, ol]
    st = lib().oracle_buildhsg_ex(
        _p(hone), _p(htwo), _p(bt), _p(bs), ctypes.c_int(nchol), _p(ref), _p(z), _p(ng), ctypes.c_int(nci),
        ctypes.c_int(CmplxConj), ctypes.c_int(ncisp), ctypes.c_int(NOcc), _p(r1), _p(r2), _p(rpg), _p(wsp),
        _p(wpg), _p(ra), _p(rb), _p(ry), ctypes.c_int(QJ), ctypes.c_int(SP), ctypes.c_int(npg), ctypes.c_int(ncipg),
        ctypes.c_int(NSO), _p(ol), ctypes.c_int(0 if ol is None else len(ol)), ctypes.c_int(nthreads),
        _p(hmat), _p(smat), _p(gmat), _p(rmat))
    if st != 0:
        raise RuntimeError(f"oracle_buildhsg failed with status {st}")
    return hmat, smat, gmat, rmat


def localg(Gradmat, Rdmmat, Smat, E0, fsp, fpg, fk, CmplxConj, NSO, nci, ncisp, ncipg):
    g, r, s = _f(Gradmat), _f(Rdmmat), _f(Smat)
    fsp_, fpg_, fk_ = (np.ascontiguousarray(np.atleast_1d(x), dtype=np.complex128) for x in (fsp, fpg, fk))
    if fk_.size < 2:
        fk_ = np.concatenate([fk_, np.zeros(2 - fk_.size, dtype=np.complex128)])
    G = np.zeros((NSO, NSO), dtype=np.complex128, order="F")
    e0 = np.complex128(E0)
    lib().oracle_localg(_p(g), _p(r), _p(s), ctypes.c_double(e0.real), ctypes.c_double(e0.imag),
                        ctypes.c_int(NSO), _p(fsp_), _p(fpg_), _p(fk_), ctypes.c_int(nci), ctypes.c_int(ncisp),
                        ctypes.c_int(ncipg), ctypes.c_int(CmplxConj), _p(G))
    return G


def num_threads() -> int:
    return int(lib().oracle_num_threads())
