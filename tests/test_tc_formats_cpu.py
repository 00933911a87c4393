"""The CPU emulation of the BF16x3 / TF32 operand formats that the GPU tests compare against:
the BF16 split represents a value to ~2^-17 relative, TF32 rounding keeps 10 fraction bits with
ties away from zero, and the scaled emulated product approaches A B^T at the expected rate."""
import numpy as np

from tests import _tc_formats as tf


def test_tf32_rounding_known_values():
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -10)
    x = np.array([1.0, 1.0 + 2.0 ** -11, 1.0 + 2.0 ** -11 - 2.0 ** -20, -(1.0 + 2.0 ** -11), 1.0 + 3 * 2.0 ** -11,
                  0.0], dtype=np.float32)
    got = tf.tf32_rna(x)
    want = np.array([one, one + ulp, one, -(one + ulp), one + 2 * ulp, 0.0], dtype=np.float32)
    assert np.array_equal(got, want), (got, want)
    assert np.all((got.view(np.uint32) & np.uint32(0x1FFF)) == 0)


def test_bf16_split_represents_value_to_16_bits():
    rng = np.random.default_rng(3)
    A = rng.normal(size=(50, 300)) * 10.0 ** rng.uniform(-4, 4, size=(50, 1))
    e, (hi, lo) = tf.parts(A, "bf16x3")
    r = np.ldexp(A, -e[:, None])
    assert np.abs(r).max() < 1.0
    assert np.abs(r - hi).max() <= 2.0 ** -8  # half a bf16 ulp of a value below 1
    assert np.abs(r - hi - lo).max() <= 2.0 ** -16
    # hi has 8 significant bits, lo is a bf16 too
    for v in (hi, lo):
        b = v.astype(np.float32).view(np.uint32)
        assert np.all((b & np.uint32(0xFFFF)) == 0)


def test_emulated_products_converge_at_the_format_precision():
    rng = np.random.default_rng(4)
    A = rng.normal(size=(40, 500))
    Bt = rng.normal(size=(30, 500))
    ref = A @ Bt.T
    scale = np.abs(A) @ np.abs(Bt).T
    e_bf = np.abs(tf.emulate(A, Bt, "bf16x3") - ref) / scale
    e_tf = np.abs(tf.emulate(A, Bt, "tf32") - ref) / scale
    e_hi = np.abs(tf.emulate(A, Bt, "bf16x3", terms=[(0, 0)]) - ref) / scale
    assert e_bf.max() < 2.0 ** -15
    assert 2.0 ** -16 < e_tf.max() < 2.0 ** -9
    assert e_hi.max() > 30 * e_bf.max()  # the cross products matter


def test_accumulation_bound_is_below_a_missing_cross_product():
    """The GPU comparison at k = 64 (bf16x3) and k = 32 (tf32) can tell a missing product term or a
    missed rounding from FP32 accumulation error."""
    rng = np.random.default_rng(5)
    A = rng.normal(size=(200, 64))
    Bt = rng.normal(size=(150, 64))
    bound = tf.accumulation_bound(A, Bt, "bf16x3")
    gap = np.abs(tf.emulate(A, Bt, "bf16x3") - tf.emulate(A, Bt, "bf16x3", terms=[(0, 0), (0, 1)]))
    assert (gap / bound).max() > 3.0
    A, Bt = A[:, :32], Bt[:, :32]
    bound = tf.accumulation_bound(A, Bt, "tf32")
    gap = np.abs(tf.emulate(A, Bt, "tf32") - A @ Bt.T)
    assert (gap / bound).max() > 3.0
