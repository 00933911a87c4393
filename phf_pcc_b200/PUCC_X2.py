"""The projected-CC grid kernel under the names of the reference's f2py module ``PUCC_X2``.

The reference compiles SUCCSD_Boson_cmplx/ into the extension ``PUCC_X2`` (Main_PCC.py:5 imports its
``pgcc`` driver).  Its grid kernel is ``PbarHbarOlap`` of the Fortran module ``fpucc``
(SUCCSD_Boson_cmplx/FPUCC.f90:14-272), which the driver calls once per Broyden iteration, followed by
``PbarHbarResFromOlap`` (:394-427).  ``fpucc.pbarhbarolap`` here takes the Fortran dummy arguments after
the six outputs, in their order, and returns the outputs (Olap0, OlapEx1, OlapEx2, EOlap0, EOlapEx1,
EOlapEx2) as f2py does; the computation runs on the GPU through libphf_b200.so.  The Broyden driver
``pgcc`` itself is not part of this library.
"""
from __future__ import annotations

import numpy as np

from . import api
from ._lib import PHFError

__all__ = ["fpucc", "PHFError"]


def _proj_sz(res1, res2, nocc, nso):
    """ProjSz (SUCCSD_Boson_cmplx/FPUCC_Tools.f90:150-169): zero the spin-flip components of vo and vvoo
    arrays, MO order [occ alpha, occ beta, vir alpha, vir beta]."""
    noa, nva = nocc // 2, nso // 2 - nocc // 2
    so = np.arange(nocc) >= noa
    sv = np.arange(nso - nocc) >= nva
    m1 = sv[:, None] == so[None, :]
    m2 = (sv[:, None, None, None].astype(int) + sv[None, :, None, None]) == (
        so[None, None, :, None].astype(int) + so[None, None, None, :])
    return np.where(m1, res1, 0), np.where(m2, res2, 0)


class _FPUCCModule:
    """Namespace mirroring the Fortran module ``fpucc``."""

    def pbarhbarolap(self, hone, htwo, ref, t1, t2, nocc, nao, nso, enuc, qj, sp, npoints, npg, ncisp, ncipg, ncik,
                     r1, r2, rpg, rk, roota, rootb, rooty, weightsp, weightpg, fsp, fpg, fk, trunode, comm=None):
        return api.pbarhbarolap(hone, htwo, ref, t1, t2, nocc, nao, nso, enuc, qj, sp, npoints, npg, ncisp, ncipg,
                                ncik, r1, r2, rpg, rk, roota, rootb, rooty, weightsp, weightpg, fsp, fpg, fk, trunode,
                                comm=comm)

    def pbarhbarresfromolap(self, ref, olap0, olapex1, olapex2, eolap0, eolapex1, eolapex2, nocc, nao, nso, sp):
        """PbarHbarResFromOlap (FPUCC.f90:394-427): Ene = EOlap0 / Olap0, Res0 = 0,
        Res1 = (EOlapEx1 - Ene OlapEx1) / Olap0, Res2 likewise (ProjSz for sp == 2).  O(v^2 o^2) host
        arithmetic on the kernel's sums."""
        del ref, nao
        ene = eolap0 / olap0
        res1 = (np.asarray(eolapex1) - ene * np.asarray(olapex1)) / olap0
        res2 = (np.asarray(eolapex2) - ene * np.asarray(olapex2)) / olap0
        if sp == 2:
            res1, res2 = _proj_sz(res1, res2, int(nocc), int(nso))
        return ene, 0j, np.asfortranarray(res1), np.asfortranarray(res2)


fpucc = _FPUCCModule()
