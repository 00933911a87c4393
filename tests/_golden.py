"""Helpers that load the golden fixtures and rebuild the arrays they do not store."""
import os

import numpy as np

from oracle import phf_oracle as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["tiny_sp1", "c1", "j1_c2v_b1", "j2_c2v_a1", "suhf_sp2_real", "cmplx2", "tiny_dense_htwo", "e_c4v",
         "j1_e_c4v"]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


def htwo_mo(case):
    """Dense <ij||kl> in the Ref-MO basis (rebuilt from the stored Cholesky vectors)."""
    if "HTwo" in case:
        return case["HTwo"]
    return orc.mo_transform_2(orc.dense_htwo_from_chol(case["B"]), case["Ref"])


def grid_kwargs(c):
    return dict(ngrid=[int(x) for x in c["ngrid"]], nci=int(c["nci"]), CmplxConj=int(c["CmplxConj"]),
                ncisp=int(c["ncisp"]), NOcc=int(c["N"]), R1=c["R1"], R2=c["R2"], Rpg=c["Rpg"],
                weightsp=c["weightsp"], weightpg=c["weightpg"], roota=c["roota"], rootb=c["rootb"],
                rooty=c["rooty"], QJ=int(c["J"]), SP=int(c["SP"]), npg=int(c["npg"]), ncipg=int(c["ncipg"]),
                NSO=int(c["M"]))
