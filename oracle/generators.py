"""Seeded synthetic inputs for the oracle and the tests.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Two generators:

* ``bm_create_synthetic_random`` restates the reference's test generator
  (src/blockmatrix.jl:878-919 for ndiag=3 and :921-964 for general ndiag): block
  sizes ``round(8*rand + b - 4)``, complex entries uniform in [0,1) for real and
  imaginary parts, off-diagonal blocks damped by 0.3.  Julia's RNG stream
  cannot be reproduced, so numpy's ``default_rng(seed)`` stands in.
* ``physics_system`` (in ``physics.py``) builds the Hermitian H / Sigma_L /
  Sigma_R systems of the benchmark configurations.
"""

import numpy as np

from .blockmatrix import BlockMatrix


def _rand_c(rng, shape):
    # Julia rand(ComplexF64, dims): real and imaginary parts uniform in [0, 1)
    return rng.random(shape) + 1j * rng.random(shape)


def random_block_sizes(rng, npl, b, uniform=False):
    if uniform:
        return [int(b)] * npl
    return [int(x) for x in np.round(8.0 * rng.random(npl) + (b - 4.0))]


def bm_create_synthetic_random(npl, b, seed=0, ndiag=3, is_hermitian=False, uniform=False,
                               block_sizes=None):
    """Random block n-diagonal BlockMatrix (blockmatrix.jl:878-964)."""
    rng = np.random.default_rng(seed)
    sizes = block_sizes if block_sizes is not None else random_block_sizes(rng, npl, b, uniform)
    bm = BlockMatrix(sizes, {"in": ndiag, "out": ndiag}, is_hermitian)
    w = (ndiag - 1) // 2
    for i in range(npl):
        if not is_hermitian:
            for j in range(i - 1, max(0, i - w) - 1, -1):
                bm.M[(i, j)] = 0.3 * _rand_c(rng, (sizes[i], sizes[j]))
        bm.M[(i, i)] = _rand_c(rng, (sizes[i], sizes[i]))
        for j in range(i + 1, min(npl, i + w + 1)):
            bm.M[(i, j)] = 0.3 * _rand_c(rng, (sizes[i], sizes[j]))
    return bm


def hermitian_random_like(bm, seed=1):
    """The Hermitian middle operator of the Keldysh test
    (test_keldyshndiag.jl:66-71): a random band matrix A, then (A + A^H)/2
    stored in Hermitian (diagonal + upper) form."""
    from .blockmatrix import bm_convert_dense, bm_from_dense
    rng = np.random.default_rng(seed)
    tmp = BlockMatrix(bm.blockSizes, bm.ndiag, False)
    w = bm.band("in")
    for i in range(bm.npl):
        for j in range(max(0, i - w), min(bm.npl, i + w + 1)):
            tmp.M[(i, j)] = _rand_c(rng, (bm.blockSizes[i], bm.blockSizes[j]))
    d = bm_convert_dense(tmp)
    d = (d + np.conj(d).T) / 2.0
    return bm_from_dense(d, bm.blockSizes, bm.ndiag, True)


def set_sparse_block(block_sizes, rind, cind, symmetric=True, seed=0, dominance=True):
    """``set_sparse_Block(b, rind, cind, s_flag)`` (src/block.jl:582-598) with
    1-based index lists; real uniform [0,1) blocks, plus ``n*I`` on the
    diagonal blocks as the selected-inverse test does
    (test_selected_inverse.jl:12-14).  Returns a dict {(i,j): float64 array}."""
    rng = np.random.default_rng(seed)
    A = {}
    for r, c in zip(rind, cind):
        i, j = r - 1, c - 1
        A[(i, j)] = rng.random((block_sizes[i], block_sizes[j]))
        if symmetric and i != j:
            A[(j, i)] = rng.random((block_sizes[j], block_sizes[i]))
    if dominance:
        n = sum(block_sizes)
        for i in range(len(block_sizes)):
            A[(i, i)] = A[(i, i)] + n * np.eye(block_sizes[i])
    return A


def full_of_blocks(A, block_sizes, dtype=np.complex128):
    """``full(A)`` (src/block.jl:547-569)."""
    off = np.concatenate([[0], np.cumsum(block_sizes)]).astype(int)
    n = off[-1]
    out = np.zeros((n, n), dtype=dtype)
    for (i, j), blk in A.items():
        out[off[i]:off[i + 1], off[j]:off[j + 1]] = blk
    return out
