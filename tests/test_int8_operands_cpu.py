"""Host-side checks of the int8 operand construction behind the batched F X product (oz_gemm_fx).

A numpy restatement of the slicing (balanced base-254 digits: r_0 = x 2^-e 127, d_t = rint(r_t),
r_{t+1} = 254 (r_t - d_t), rint to nearest even) and of the operands: X's columns as rows of 2M reals
(Re, Im interleaved over i), each complex row c of F as two rows (Re F[c][i], -Im F[c][i]) and
(Im F[c][i], Re F[c][i]).  Checked: the digits of -x are the negated digits of x (the slicer of F's
rows forms Re's and Im's digits once and negates them), the real dot products give Re and Im of F X,
the little-endian packing of a row's digit pairs into 2- and 4-byte words, and the error of the
product from the sliced operands (group sums t + u < S, as the GEMM keeps them) against its bound.
Test infrastructure only: no device call.
"""
import numpy as np

S = 5


def exponents(A):
    """e_i with max|A_i.| = f 2^e_i, f in [0.5, 1) (frexp), 0 for a zero row."""
    mx = np.abs(A).max(axis=1)
    _, e = np.frexp(mx)
    return np.where(mx > 0, e, 0).astype(np.int64)


def digits(A, e, s=S):
    """Slices of the rows of A at row exponents e: int array (s, rows, k)."""
    r = np.ldexp(A, -e[:, None]) * 127.0
    out = []
    for _ in range(s):
        d = np.rint(r)
        out.append(d.astype(np.int64))
        r = (r - d) * 254.0
    return np.array(out)


def sliced_product(A, B, s=S):
    """A B^T from the slices of A's and B's rows, keeping the digit products t + u < s (0-based)."""
    ea, eb = exponents(A), exponents(B)
    da, db = digits(A, ea, s), digits(B, eb, s)
    acc = np.zeros((A.shape[0], B.shape[0]))
    for t in range(s):
        for u in range(s - t):
            acc += (da[t] @ db[u].T).astype(np.float64) * 254.0 ** -(t + u)
    return np.ldexp(acc / (127.0 * 127.0), ea[:, None] + eb[None, :])


def fx_operands(F, X):
    """The A operand (N rows of 2M: X's columns) and the B operand (2M rows of 2M: F's rows)."""
    M, N = X.shape
    A = np.empty((N, 2 * M))
    A[:, 0::2], A[:, 1::2] = X.real.T, X.imag.T
    B = np.empty((2 * M, 2 * M))
    B[0::2, 0::2], B[0::2, 1::2] = F.real, -F.imag
    B[1::2, 0::2], B[1::2, 1::2] = F.imag, F.real
    return A, B


def test_digits_are_balanced_and_odd_in_x():
    rng = np.random.default_rng(5)
    A = rng.normal(size=(40, 300)) * 10.0 ** rng.uniform(-6, 6, size=(40, 1))
    e = exponents(A)
    d, dn = digits(A, e), digits(-A, e)
    assert np.abs(d).max() <= 127
    assert np.array_equal(dn, -d)
    back = np.ldexp(sum(d[t] * 254.0 ** -t for t in range(S)) / 127.0, e[:, None])
    assert (np.abs(back - A) / np.ldexp(1.0, e)[:, None]).max() <= 254.0 ** -S


def test_fock_rows_and_orbital_columns_give_the_complex_product():
    rng = np.random.default_rng(6)
    M, N = 24, 7
    F = rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))
    X = rng.normal(size=(M, N)) + 1j * rng.normal(size=(M, N))
    A, B = fx_operands(F, X)
    Dt = A @ B.T  # row j, column 2c + part
    FX = F @ X
    assert np.abs(Dt[:, 0::2] - FX.real.T).max() <= 1e-12 * np.abs(FX).max()
    assert np.abs(Dt[:, 1::2] - FX.imag.T).max() <= 1e-12 * np.abs(FX).max()
    # both Fock rows of c share one exponent: the largest |Re| or |Im| of F's row c
    eb = exponents(B)
    assert np.array_equal(eb[0::2], eb[1::2])


def test_packed_digit_pairs_decode_to_the_row_bytes():
    rng = np.random.default_rng(7)
    dr = rng.integers(-127, 128, size=64)
    di = rng.integers(-127, 128, size=64)
    # 2-byte words (one element per lane) and 4-byte words (two elements per lane), little-endian
    u0 = (dr & 0xFF) | ((-di & 0xFF) << 8)
    u1 = (di & 0xFF) | ((dr & 0xFF) << 8)
    row_r = np.frombuffer(u0.astype("<u2").tobytes(), dtype=np.int8)
    row_r1 = np.frombuffer(u1.astype("<u2").tobytes(), dtype=np.int8)
    assert np.array_equal(row_r[0::2], dr) and np.array_equal(row_r[1::2], -di)
    assert np.array_equal(row_r1[0::2], di) and np.array_equal(row_r1[1::2], dr)
    w0 = u0[0::2].astype(np.uint64) | (u0[1::2].astype(np.uint64) << 16)
    w1 = u1[0::2].astype(np.uint64) | (u1[1::2].astype(np.uint64) << 16)
    assert np.array_equal(np.frombuffer(w0.astype("<u4").tobytes(), dtype=np.int8), row_r)
    assert np.array_equal(np.frombuffer(w1.astype("<u4").tobytes(), dtype=np.int8), row_r1)


def test_sliced_fx_product_meets_its_bound():
    rng = np.random.default_rng(8)
    M, N = 40, 9
    F = (rng.normal(size=(M, M)) + 1j * rng.normal(size=(M, M))) * 10.0 ** rng.uniform(-2, 2, size=(M, 1))
    X = rng.normal(size=(M, N)) + 1j * rng.normal(size=(M, N))
    A, B = fx_operands(F, X)
    got = sliced_product(A, B)
    exact = A @ B.T
    scale = np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=1)[None, :]
    k = A.shape[1]
    assert (np.abs(got - exact) / scale).max() <= (S + 1) * k * 254.0 ** -S
