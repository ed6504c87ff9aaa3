"""CPU model of the library's mixed-precision complex products (NEGF_PREC_MIXED:
FP64-grade products from INT8 digit products on the tensor cores).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): nothing in the library
imports it.  It restates, in numpy, the arithmetic of the digit split and the
digit-pair products of ``libnegf.jl_b200/csrc/zgemm_ozaki.cu`` so that the
accuracy those products claim can be checked on the host against an exact
(double-double) product, independently of the GPU.  The reference (LibNEGF.jl)
computes in ComplexF64 only; this part has no counterpart there.

The scheme is Ozaki's error-free splitting (Ozaki, Ogita, Oishi and Rump,
"Error-free transformations of matrix multiplication by using fast routines
of matrix multiplication and its applications", 2012) in its integer form
(Ootomo, Ozaki and Yokota, "DGEMM on integer matrix multiplication unit",
2024), as the library applies it to a complex product C = op(A) op(B):

* every row r of an operand view Y (left: the rows of op(A); right: the
  columns of op(B), both K long) gets one exponent e_r with
  max_k |Re Y| + |Im Y| < 2^e_r (0 for a zero row), shared by its real part,
  its imaginary part and their sum (the three real operands of Gauss's 3M
  product);
* x = rint(y 2^(54 - e_r)) is an integer with |x| <= 2^54 (the sum
  xr + xi as well); it is written as seven balanced base-256 digits,
  x = sum_i s_i 256^(6 - i), the six lower ones in [-128, 127] and the top
  one in [-64, 64], read as the bytes of x + C6 with C6 = 128 (256^6 - 1)/255;
* a real product is sum_D 2^(e_A + e_B - 12 - 8D) acc_D, where acc_D is the
  exact integer sum over k and over the digit pairs i + j = D, D <= 7 (34
  pairs) or D <= 6 (28 pairs);
* complex: P1 = Ar Br, P2 = Ai Bi, P3 = (Ar + Ai)(Br + Bi), Re C = P1 - P2,
  Im C = P3 - P1 - P2.
"""

import numpy as np

NDIG = 7  # base-256 digits per 54-bit value
C6 = 128 * (256 ** 6 - 1) // 255


def row_exponents(Y):
    """e_r with max_k |Re Y[r,k]| + |Im Y[r,k]| < 2^e_r (0 for a zero row)."""
    mx = np.max(np.abs(Y.real) + np.abs(Y.imag), axis=1) if Y.shape[1] else np.zeros(Y.shape[0])
    _, e = np.frexp(mx)
    return np.where(mx > 0, e, 0).astype(np.int64)


def fixed_point(Y, e, conj=False):
    """The three 54-bit integers (Re, Im, Re + Im) of Y's rows at scale
    2^(54 - e_r); conj takes the conjugate of Y."""
    f = np.ldexp(1.0, (54 - e))[:, None]
    xr = np.rint(Y.real * f).astype(np.int64)
    xi = np.rint((-Y.imag if conj else Y.imag) * f).astype(np.int64)
    return xr, xi, xr + xi


def digits(x):
    """Seven balanced base-256 digits s_0 (top) .. s_6 of the int64 array x
    (|x| <= 2^54): the bytes of x + C6, the lower six minus 128.  Returned as
    float64 arrays (exact small integers)."""
    u = x + np.int64(C6)
    out = [(u >> np.int64(48)).astype(np.float64)]  # arithmetic shift: the top digit with its sign
    for b in range(5, -1, -1):
        out.append((((u >> np.int64(8 * b)) & np.int64(255)) - 128).astype(np.float64))
    return out


def digit_pairs(pairs):
    """Digit diagonals D kept: 0..7 for 34 pairs, 0..6 for 28."""
    if pairs not in (28, 34):
        raise ValueError("pairs must be 28 or 34")
    return 7 if pairs == 28 else 8


def real_product(dA, eA, dB, eB, pairs):
    """sum_k A[r,k] B[c,k] from the digits of A's rows (dA) and B's rows (dB):
    the exact diagonal sums acc_D (float64 BLAS products of small integers
    are exact: |acc_D| <= 7 K 2^14 < 2^53), then the FP64 sum of
    acc_D 2^(-12 - 8D) scaled by 2^(e_A + e_B).  Also returns
    sum_D |acc_D| 2^(-12 - 8D), the scale of that sum's rounding."""
    nd = digit_pairs(pairs)
    val = np.zeros((dA[0].shape[0], dB[0].shape[0]))
    mag = np.zeros_like(val)
    for D in range(nd):
        acc = np.zeros_like(val)
        for i in range(max(0, D - (NDIG - 1)), min(D, NDIG - 1) + 1):
            acc += dA[i] @ dB[D - i].T
        w = 2.0 ** (-12 - 8 * D)
        val += acc * w
        mag += np.abs(acc) * w
    s = np.ldexp(1.0, (eA[:, None] + eB[None, :]).astype(np.int64))
    return val * s, mag * s


def zgemm(A, B, pairs=34, opA="N", opB="N"):
    """op(A) op(B) as the library's mixed path forms it (op: N, T or C).
    Returns (C, info): info holds the row exponents and, per real product,
    the rounding scale of its FP64 diagonal sum (for error_bound)."""
    op = {"N": lambda x: x, "T": lambda x: x.T, "C": lambda x: x.T}
    YA = op[opA](np.asarray(A, dtype=np.complex128))       # m x K
    YB = op[opB](np.asarray(B, dtype=np.complex128)).T     # n x K (rows of op(B)^T)
    eA, eB = row_exponents(YA), row_exponents(YB)
    xa = fixed_point(YA, eA, conj=opA == "C")
    xb = fixed_point(YB, eB, conj=opB == "C")
    P, mags = [], []
    for p in range(3):
        v, m = real_product(digits(xa[p]), eA, digits(xb[p]), eB, pairs)
        P.append(v)
        mags.append(m)
    C = (P[0] - P[1]) + 1j * (P[2] - P[0] - P[1])
    return C, {"eA": eA, "eB": eB, "P": P, "mag": mags, "K": YA.shape[1], "pairs": pairs}


def dropped_per_k(pairs):
    """Bound of the digit pairs a product leaves out, per k, relative to
    2^(e_A + e_B): pairs on diagonal D contribute at most
    |s_i s_j| 256^(12 - D) 2^-108 <= 2^(2 - 8D) each, and D >= 7 has 13 - D
    pairs."""
    nd = digit_pairs(pairs)
    return sum((13 - D) * 2.0 ** (2 - 8 * D) for D in range(nd, 13))


def error_bound(info):
    """Rigorous elementwise bounds (Re, Im) of |C_model - C_exact| for zgemm's
    result.  Per real product, K 2^(e_A + e_B) times the operand rounding
    (|x| <= 2^54 and a rounding error of 1/2 per operand: 2^-54; the 3M sum
    xr + xi carries two roundings: 2^-53) plus the dropped pairs; then the
    rounding of its FP64 diagonal sum (ND u sum_D |acc_D| w_D) and that of
    the 3M combination."""
    u = 2.0 ** -53
    K, nd = info["K"], digit_pairs(info["pairs"])
    s = np.ldexp(1.0, (info["eA"][:, None] + info["eB"][None, :]).astype(np.int64))
    drop = dropped_per_k(info["pairs"])
    e = [K * s * (rep + 2.0 ** -106 + drop) + nd * u * m
         for rep, m in zip((2.0 ** -54, 2.0 ** -54, 2.0 ** -53), info["mag"])]
    P = [np.abs(x) for x in info["P"]]
    re = e[0] + e[1] + u * (P[0] + P[1])
    im = e[0] + e[1] + e[2] + 2 * u * (P[0] + P[1] + P[2])
    return re, im
