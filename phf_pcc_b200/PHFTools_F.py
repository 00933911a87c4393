"""Drop-in for the reference's f2py module ``PHFTools_F`` (PHF_fort/makefile:7).

``from phf_pcc_b200.PHFTools_F import phftools`` gives an object whose ``buildhsg`` and
``localg`` take the positional arguments PHF.py passes (PHF.py:44-45, :70-71, :76) and
return what the f2py wrappers return: Fortran-ordered complex128 arrays
(Hmat, Smat, Gradmat, Rdmmat) and the (nso, nso) G.  Dimension arguments that f2py makes
optional (npg, ncipg, nso, nci, ncisp, ncipg) are inferred from the array shapes when
omitted.  The computation runs on the GPU through libphf_b200.so.

Where the Fortran executes ``STOP`` (PHFTools.f90:199, Wrappers.f90:226,311,328) this
module raises ``PHFError`` (a RuntimeError).  ``phftools.on_not_hermitian = "return"``
returns the non-Hermitian result instead of raising.

``comm`` is accepted and not used: the reference's MPI split over grid points is commented
out (PHFTools.f90:85-86), so every rank sums the whole grid and MPI_reduce multiplies
Hmat, Smat, Gradmat and Rdmmat by the number of ranks (the energy and G are unchanged).
One process per GPU evaluates the whole grid here.
"""
from __future__ import annotations

from . import api
from ._lib import PHFError

__all__ = ["phftools", "PHFError"]


class _PHFToolsModule:
    """Namespace mirroring the Fortran module ``phftools``."""

    on_not_hermitian = "raise"

    def buildhsg(self, hone, htwo, ref, z, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg,
                 roota, rootb, rooty, qj, sp, comm=None, npg=None, ncipg=None, nso=None):
        return api.buildhsg(hone, htwo, ref, z, ngrid, nci, cmplxconj, ncisp, nocc, r1, r2, rpg, weightsp, weightpg,
                            roota, rootb, rooty, qj, sp, npg=npg, ncipg=ncipg, nso=nso,
                            check_hermitian=(self.on_not_hermitian == "raise"))

    def localg(self, gradmat, rdmmat, smat, e0, fsp, fpg, fk, cmplxconj, nso=None, nci=None, ncisp=None,
               ncipg=None):
        return api.localg(gradmat, rdmmat, smat, e0, fsp, fpg, fk, cmplxconj, nso=nso, nci=nci, ncisp=ncisp,
                          ncipg=ncipg)


    def buildsc(self, c0, c1, c2, nocc, ngrid, qj, r1, r2, rpg, rk, roota, rootb, rooty, weightsp, weightpg, fsp,
                fpg, fk, nso=None, npg=None, ncisp=None, ncipg=None, ncik=None):
        """BuildSC (PHF_fort/PHFTools.f90:464-537) with the f2py argument order of its Fortran dummy
        arguments (outputs t0, t1, t2 returned; dimensions optional).  The reference's LinDep.py:73
        passes a different list (it inserts ``nci`` after ``J``), which does not match that Fortran
        routine; this follows the Fortran."""
        return api.buildsc(c0, c1, c2, nocc, ngrid, qj, r1, r2, rpg, rk, roota, rootb, rooty, weightsp, weightpg,
                           fsp, fpg, fk, nso=nso, npg=npg, ncisp=ncisp, ncipg=ncipg, ncik=ncik)


phftools = _PHFToolsModule()
