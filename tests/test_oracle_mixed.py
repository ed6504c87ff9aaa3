"""The mixed-precision product arithmetic on the host: the digit split and the
digit-pair products of the library's INT8 path (oracle/ozaki.py restates
them) against an exact double-double product (oracle/ddtruth.py).

What is pinned here:
* the split is exact where it claims to be: seven balanced base-256 digits
  (read as the bytes of x + C6) reconstruct every 54-bit x, within the digit
  ranges an int8 operand holds, and rounding to 54 bits errs by at most
  2^(e_r - 55);
* every product, for all op pairs, ragged K and rows of very different
  magnitudes (and zero rows), lies within the rigorous elementwise bound of
  the scheme (operand rounding + dropped digit pairs + FP64 summation);
* the two accuracy levels the library states: 34 pairs are as accurate as an
  FP64 GEMM, 28 pairs stay near 1e-15 relative to |op(A)| |op(B)|.
"""

import numpy as np
import pytest

from oracle import ddtruth, ozaki


def _exact(A, B):
    t = ddtruth.matmul(ddtruth.DD(A), ddtruth.DD(B))
    return t.hi, t.lo


def _err(C, hi, lo):
    """|C - (hi + lo)| per part, without rounding hi + lo first."""
    return np.abs((C.real - hi.real) - lo.real), np.abs((C.imag - hi.imag) - lo.imag)


def _operands(rng, m, K, n, spread=6.0):
    A = (rng.standard_normal((m, K)) + 1j * rng.standard_normal((m, K))) * np.exp(rng.uniform(-spread, spread, (m, 1)))
    B = (rng.standard_normal((K, n)) + 1j * rng.standard_normal((K, n))) * np.exp(rng.uniform(-spread, spread, (1, n)))
    A[min(3, m - 1)] = 0.0  # a zero row: exponent 0, all digits zero
    return A, B


def test_digits_reconstruct_every_54_bit_value():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.integers(-2 ** 54, 2 ** 54, 20000, endpoint=True, dtype=np.int64),
                        np.array([0, 1, -1, 2 ** 54, -2 ** 54, 2 ** 48 - 1, -2 ** 48, 127, -128, 128, -129],
                                 dtype=np.int64)])
    d = ozaki.digits(x)
    assert len(d) == ozaki.NDIG
    assert np.all(np.abs(d[0]) <= 64)
    for s in d[1:]:
        assert np.all((s >= -128) & (s <= 127))
    back = [sum(int(d[i][k]) * 256 ** (6 - i) for i in range(ozaki.NDIG)) for k in range(len(x))]
    assert back == [int(v) for v in x]


def test_fixed_point_rounding():
    rng = np.random.default_rng(1)
    Y = (rng.standard_normal((50, 70)) + 1j * rng.standard_normal((50, 70))) * np.exp(rng.uniform(-20, 20, (50, 1)))
    Y[7] = 0.0
    e = ozaki.row_exponents(Y)
    mx = np.max(np.abs(Y.real) + np.abs(Y.imag), axis=1)
    assert np.all(mx < np.ldexp(1.0, e)) and np.all(mx[mx > 0] >= np.ldexp(0.5, e[mx > 0]))
    for conj in (False, True):
        xr, xi, xs = ozaki.fixed_point(Y, e, conj)
        for x in (xr, xi, xs):
            assert np.all(np.abs(x) <= 2 ** 54)
        scale = np.ldexp(1.0, e - 54)[:, None]
        half = np.ldexp(1.0, e - 55)[:, None]
        assert np.all(np.abs(xr * scale - Y.real) <= half)
        assert np.all(np.abs(xi * scale - (-Y.imag if conj else Y.imag)) <= half)


@pytest.mark.parametrize("pairs", [34, 28])
@pytest.mark.parametrize("K", [1, 29, 256, 1024])
@pytest.mark.parametrize("ops", ["NN", "NC", "CN", "TN", "NT", "CC"])
def test_products_within_the_rigorous_bound(pairs, K, ops):
    rng = np.random.default_rng(K * 7 + pairs + 3 * "NTC".index(ops[0]) + "NTC".index(ops[1]))
    m, n = 37, 21
    A, B = _operands(rng, m, K, n)
    opA, opB = ops
    Ain = A if opA == "N" else (A.T if opA == "T" else A.conj().T)
    Bin = B if opB == "N" else (B.T if opB == "T" else B.conj().T)
    C, info = ozaki.zgemm(Ain, Bin, pairs, opA, opB)
    hi, lo = _exact(A, B)
    er, ei = _err(C, hi, lo)
    br, bi = ozaki.error_bound(info)
    assert np.all(er <= br) and np.all(ei <= bi)
    assert np.all(C[3] == 0.0)


def test_accuracy_levels():
    """At the contraction lengths of the solver's products (K = 256) and the
    long ones the mixed GEMM primitive accepts (K = 1024): 34 pairs no less
    accurate than an FP64 GEMM (elementwise, relative to |A||B|), 28 pairs
    within 1.5e-15 of |A||B| (the ~1e-15 the header states) and bounded by
    3 K u 2^(e_A + e_B), three times the FP64 rounding bound at the row
    scales."""
    rng = np.random.default_rng(11)
    u = 2.0 ** -53
    for K in (256, 1024):
        A, B = _operands(rng, 48, K, 40, spread=3.0)
        hi, lo = _exact(A, B)
        absAB = np.abs(A) @ np.abs(B)
        nz = absAB > 0
        fp = A @ B
        e_fp = np.abs((fp - hi) - lo)[nz] / absAB[nz]
        for pairs in (34, 28):
            C, info = ozaki.zgemm(A, B, pairs)
            e = np.abs((C - hi) - lo)
            rel = e[nz] / absAB[nz]
            scale = K * u * np.ldexp(1.0, info["eA"][:, None] + info["eB"][None, :])
            if pairs == 34:
                assert rel.max() <= max(1.5 * e_fp.max(), 2 * u)
            else:
                assert rel.max() < 1.5e-15
                assert np.all(e <= 3.0 * scale)
