"""Oracle restatement of LibNEGF.jl's CPU backend primitives.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Every function maps one ``be_*`` call of ``src/backend_cpu.jl`` onto the same
LAPACK/BLAS routine through scipy (which bundles OpenBLAS; the reference pins
OpenBLAS_jll 0.3.29 through libblastrampoline).  Blocks are complex128 numpy
arrays; an LU is the pair ``(factors, ipiv)`` exactly as ``CpuLU`` holds it
(``backend_cpu.jl:7-10``), with 0-based pivots.
"""

import numpy as np
from scipy.linalg import blas, lapack


class LinAlgError(RuntimeError):
    """Raised where the reference prints an error and calls ``exit()``."""


def be_lu(A):
    """``be_lu!`` (backend_cpu.jl:147-169): zgetrf on a copy of A.

    The reference prints and exits on ``info != 0``; here an exception."""
    lu, piv, info = lapack.zgetrf(np.asarray(A, dtype=np.complex128))
    if info != 0:
        raise LinAlgError("LAPACK lu returned an error info %d" % info)
    return (lu, piv)


def be_mldivide(trans, B, LU):
    """``be_mldivide!`` (backend_cpu.jl:193-206): zgetrs with trans 'N' or 'C'."""
    lu, piv = LU
    t = {"N": 0, "T": 1, "C": 2}[trans]
    x, info = lapack.zgetrs(lu, piv, np.asarray(B, dtype=np.complex128), trans=t)
    if info != 0:
        raise LinAlgError("getrs info %d" % info)
    return x


def _op_flag(t):
    return {"N": 0, "T": 1, "C": 2}[t]


def be_gemm(tA, tB, alpha, A, B, beta, C):
    """``be_gemm!`` (backend_cpu.jl:208-219): zgemm; returns the new C."""
    if C is None:
        C = np.zeros((A.shape[1] if tA != "N" else A.shape[0],
                      B.shape[0] if tB != "N" else B.shape[1]), dtype=np.complex128)
    return blas.zgemm(alpha, A, B, beta=beta, c=np.asfortranarray(C, dtype=np.complex128),
                      trans_a=_op_flag(tA), trans_b=_op_flag(tB), overwrite_c=0)


def be_ctranspose(A):
    """``be_ctranspose!`` (backend_cpu.jl:58-68)."""
    return np.ascontiguousarray(np.conj(A).T)


def be_getrf(A):
    """``be_getrf!`` (backend_cpu.jl:255-265): zgetrf, pivots DISCARDED.

    The selected-inverse path calls LAPACK getrf and throws the pivot vector
    away (``selected_inverse.jl:18``), so the returned factors are those of
    P*A while later steps use them as if P = I."""
    lu, _piv, info = lapack.zgetrf(np.asarray(A, dtype=np.complex128))
    return lu


def lu_nopivot(A):
    """lu(A, NoPivot()) -- the factorisation ``selected_inverse.jl:17`` names and
    ``test_selected_inverse.jl`` checks against -- as packed L\\U factors
    (unit lower L), by right-looking elimination in blocks of 32 columns."""
    F = np.array(A, dtype=np.complex128)
    n = F.shape[0]
    nb = 32
    for k0 in range(0, n, nb):
        k1 = min(n, k0 + nb)
        for k in range(k0, k1):
            F[k + 1:, k] /= F[k, k]
            F[k + 1:, k + 1:k1] -= np.outer(F[k + 1:, k], F[k, k + 1:k1])
        if k1 < n:
            L11 = np.tril(F[k0:k1, k0:k1], -1) + np.eye(k1 - k0)
            F[k0:k1, k1:] = blas.ztrsm(1.0, L11, F[k0:k1, k1:], side=0, lower=1, diag=1)
            F[k1:, k1:] -= F[k1:, k0:k1] @ F[k0:k1, k1:]
    return F


def be_trsm(side, ul, tA, dA, alpha, A, B):
    """``be_trsm!`` (backend_cpu.jl:241-253): ztrsm."""
    return blas.ztrsm(alpha, A, np.asarray(B, dtype=np.complex128),
                      side=0 if side == "L" else 1, lower=1 if ul == "L" else 0,
                      trans_a=_op_flag(tA), diag=1 if dA == "U" else 0)


def be_getri(A):
    """``be_getri!`` (backend_cpu.jl:229-239): zgetri with identity pivots."""
    n = A.shape[0]
    inv, info = lapack.zgetri(np.asarray(A, dtype=np.complex128), np.arange(n, dtype=np.int32))
    if info != 0:
        raise LinAlgError("getri info %d" % info)
    return inv


def be_identity(n):
    """``be_identity`` (backend_cpu.jl:54-56)."""
    return np.eye(n, dtype=np.complex128)
