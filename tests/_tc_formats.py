"""CPU emulation of the floating-point operand formats of the tensor-core GEMM (phf_tc_dgemm with
PHF_PREC_BF16X3 / PHF_PREC_TF32, and the J/K contractions of plans in those precisions): the
power-of-two scaling of each operand row, the BF16 high/low split (torch's float32 -> bfloat16
conversion, round to nearest even) and the TF32 rounding (10 fraction bits, ties away from zero),
followed by exact FP64 products of the converted operands.  What the device adds on top is the
FP32 accumulation of those products.  Test infrastructure only.
"""
import numpy as np

U32 = 2.0 ** -24  # unit roundoff of FP32


def row_exponents(A):
    """e_i with max|A_i.| = f 2^e_i, f in [0.5, 1) (frexp), 0 for a zero row."""
    mx = np.abs(A).max(axis=1)
    _, e = np.frexp(mx)
    return np.where(mx > 0, e, 0).astype(np.int64)


def bf16_rn(x):
    """float32 values rounded to bfloat16 (nearest, ties to even), returned as float32."""
    import torch

    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32))
    return t.to(torch.bfloat16).to(torch.float32).numpy()


def tf32_rna(x):
    """float32 values rounded to 10 fraction bits, ties away from zero (low 13 bits cleared)."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def parts(A, fmt):
    """Row exponents and the converted parts of A scaled by 2^-e: [hi, lo] (bf16x3) or [t] (tf32)."""
    e = row_exponents(A)
    r = np.ldexp(A, -e[:, None])
    if fmt == "tf32":
        return e, [tf32_rna(r.astype(np.float32)).astype(np.float64)]
    hi = bf16_rn(r.astype(np.float32)).astype(np.float64)
    lo = bf16_rn((r - hi).astype(np.float32)).astype(np.float64)
    return e, [hi, lo]


def emulate(A, Bt, fmt, terms=None):
    """A Bt^T from the converted operands with exact FP64 products.  bf16x3 uses the products
    (hi, hi), (hi, lo), (lo, hi) unless `terms` names others; tf32 the one product."""
    ea, pa = parts(A, fmt)
    eb, pb = parts(Bt, fmt)
    if fmt == "tf32":
        terms = [(0, 0)]
    elif terms is None:
        terms = [(0, 0), (0, 1), (1, 0)]
    s = sum(pa[i] @ pb[j].T for i, j in terms)
    return np.ldexp(s, ea[:, None] + eb[None, :])


def accumulation_bound(A, Bt, fmt):
    """Worst-case FP32 accumulation error of the device sums: k 2^-23 sum_k |a'_ik||b'_jk|
    (k additions, each off by at most one FP32 ulp, directed rounding included), scaled back."""
    ea, pa = parts(A, fmt)
    eb, pb = parts(Bt, fmt)
    k = A.shape[1]
    s = np.abs(pa[0]) @ np.abs(pb[0]).T
    return np.ldexp(2.0 * k * U32 * s, ea[:, None] + eb[None, :])
