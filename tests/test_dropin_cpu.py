"""The reference's own driver imports the drop-in module unchanged (no GPU needed).

PHF.py:10 reads ``from PHFTools_F import phftools``.  With ``dropin/`` on the import path that
line must resolve to this library's ``phftools``, and an ``EandG`` call must reach it -- where,
without a GPU, the library refuses loudly instead of computing on the CPU.  Needs the reference
checkout (``PHF_REFERENCE_DIR``, default /root/reference); skipped when it is absent.
"""
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("PHF_REFERENCE_DIR", "/root/reference")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "PHF.py")), reason="reference checkout not present")
def test_reference_driver_resolves_the_dropin(tmp_path):
    code = textwrap.dedent(f"""
        import sys
        import numpy as np
        sys.path.insert(0, {ROOT!r})
        from tests._golden import htwo_mo, load
        from tests.golden.make_dropin_trace import stub_modules
        c = load("c1")
        stub_modules(c)
        sys.path.insert(0, {os.path.join(ROOT, "dropin")!r})
        sys.path.insert(0, {REF!r})
        import PHF                                   # the reference driver, unmodified
        from phf_pcc_b200.PHFTools_F import phftools
        assert PHF.phftools is phftools, "PHF.py:10 did not resolve to the drop-in"
        from phf_pcc_b200._lib import PHFError
        z = c["Z"].reshape(-1)
        try:
            PHF.EandG(np.concatenate([z.real, z.imag]), c["HOne"], htwo_mo(c), c["Ref"], 0)
        except (PHFError, ImportError) as e:
            print("REFUSED", type(e).__name__, e)
        else:
            import torch
            assert torch.cuda.is_available(), "computed without a GPU"
            print("COMPUTED")
    """)
    r = subprocess.run([sys.executable, "-c", code], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert "REFUSED" in r.stdout or "COMPUTED" in r.stdout, r.stdout
