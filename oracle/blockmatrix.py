"""Oracle restatement of LibNEGF.jl's ``BlockMatrix`` container.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

``BlockMatrix`` (src/blockmatrix.jl:10-17) holds a banded block matrix: only
blocks with |i-j| <= (ndiag-1)/2 are assigned; a Hermitian matrix stores the
diagonal and upper blocks only (blockmatrix.jl:47-56).  Indices here are
0-based; blocks live in a dict keyed by (i, j).
"""

import numpy as np


class BlockMatrix:
    def __init__(self, block_sizes, ndiag=None, is_hermitian=False):
        self.blockSizes = [int(b) for b in block_sizes]
        self.ndiag = dict(ndiag or {"in": 3, "out": 3})
        self.isHermitian = bool(is_hermitian)
        self.M = {}

    @property
    def npl(self):
        return len(self.blockSizes)

    def offsets(self):
        return np.concatenate([[0], np.cumsum(self.blockSizes)]).astype(int)

    def band(self, key="out"):
        return (self.ndiag[key] - 1) // 2

    def pattern(self, key="out"):
        """Assigned (i, j) pairs in the order bm_convert visits them
        (blockmatrix.jl:44-69)."""
        w = self.band(key)
        out = []
        for i in range(self.npl):
            if not self.isHermitian:
                for j in range(i - 1, max(0, i - w) - 1, -1):
                    out.append((i, j))
            out.append((i, i))
            for j in range(i + 1, min(self.npl, i + w + 1)):
                out.append((i, j))
        return out


def bm_from_dense(A, block_sizes, ndiag, is_hermitian=False):
    """``bm_convert(sparse, blockSizes, ndiag, isHermitian)`` (blockmatrix.jl:34-72)."""
    bm = BlockMatrix(block_sizes, ndiag, is_hermitian)
    off = bm.offsets()
    for (i, j) in bm.pattern("out"):
        bm.M[(i, j)] = np.array(A[off[i]:off[i + 1], off[j]:off[j + 1]], dtype=np.complex128)
    return bm


def bm_convert_dense(bm):
    """``bm_convert(BlockMatrix)`` (blockmatrix.jl:82-127), dense result.

    For a Hermitian matrix the lower blocks are filled with the conjugate
    transpose of the stored upper blocks (blockmatrix.jl:101-105)."""
    off = bm.offsets()
    n = off[-1]
    A = np.zeros((n, n), dtype=np.complex128)
    w = bm.band("out")
    for i in range(bm.npl):
        for j in range(max(0, i - w), min(bm.npl, i + w + 1)):
            if j < i and bm.isHermitian:
                A[off[i]:off[i + 1], off[j]:off[j + 1]] = np.conj(bm.M[(j, i)]).T
            else:
                A[off[i]:off[i + 1], off[j]:off[j + 1]] = bm.M[(i, j)]
    return A


def bm_copy(bm):
    """``bm_copy`` (blockmatrix.jl:231-262)."""
    out = BlockMatrix(bm.blockSizes, bm.ndiag, bm.isHermitian)
    out.M = {k: v.copy() for k, v in bm.M.items()}
    return out


def bm_fuse_to_tridiagonal(bm):
    """``bm_fuse_to_tridiagonal`` (blockmatrix.jl:1075-1106): fuse groups of w
    consecutive layers so that a block (2w+1)-diagonal matrix becomes block
    tridiagonal, through a dense round trip."""
    w = bm.band("in")
    if w <= 1:
        return bm_copy(bm)
    new_npl = -(-bm.npl // w)
    new_sizes = [0] * new_npl
    for ix in range(bm.npl):
        new_sizes[ix // w] += bm.blockSizes[ix]
    dense = bm_convert_dense(bm)
    return bm_from_dense(dense, new_sizes, {"in": 3, "out": 3}, bm.isHermitian)


def band_of_dense(A, block_sizes, ndiag, is_hermitian=False):
    """The band of a dense matrix as a dense matrix (zero outside the band):
    ``bm_convert(bm_convert(sparse(A), sizes, ndiag, h))`` in the reference tests."""
    return bm_convert_dense(bm_from_dense(A, block_sizes, ndiag, is_hermitian))
