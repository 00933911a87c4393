"""Drop-in for the reference's f2py extension module ``PHFTools_F`` (built by PHF_fort/makefile:7).

With this directory on ``PYTHONPATH``, the reference driver's own import line

    from PHFTools_F import phftools          # PHF.py:10

resolves to the B200 library without any edit to the driver: ``phftools.buildhsg`` and
``phftools.localg`` take the positional arguments of PHF.py:44-45, :70-71 and :76 and return what
the f2py wrappers return (see phf_pcc_b200/PHFTools_F.py, which this module re-exports).
"""
import os
import sys

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from phf_pcc_b200.PHFTools_F import PHFError, phftools  # noqa: E402

__all__ = ["phftools", "PHFError"]
