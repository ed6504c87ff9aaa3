"""CPU tests of the host-side mirror of the reference's DDRGF setup and
helpers: permutation vectors and the permuted matrix
(matinvertndiag_ddrgf_utils.jl:478-624; the reference test checks the
permuted block matrix against P M P^T, test_matinvertndiag_ddrgf.jl:84-104),
the cost-model pieces (:221-276, :455-465) against the oracle's restatement,
bm_reference! and build_M_from_HS.  Nothing here launches a kernel."""

import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT
from oracle import ddrgf as o_dd

sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
import libnegf_b200 as negf  # noqa: E402


@pytest.mark.parametrize("npl,d1", [(20, 4), (18, 3), (40, 6), (8, 1), (128, 15), (33, 2), (64, 15), (17, 3)])
def test_permutation_vector_matches_partition(npl, d1):
    nr, _ = o_dd.get_nr_tasks(npl, d1)
    if nr < 1:
        with pytest.raises(ValueError):
            negf.bndiag_of_inv_ddrgf_create_permutation_vector(npl, d1)
        return
    perm_inv, sizes = negf.bndiag_of_inv_ddrgf_create_permutation_vector(npl, d1)
    seps, doms, o_perm = o_dd.partition(npl, d1)
    assert perm_inv == o_perm
    assert sizes == [1] * len(seps) + [len(d) for d in doms]
    assert sorted(perm_inv) == list(range(npl))
    perm = negf.bndiag_of_inv_ddrgf_transpose_permutation_vector(perm_inv)
    assert [perm[p] for p in perm_inv] == list(range(npl))


def _dense(bm):
    off = bm.offsets()
    D = np.zeros((off[-1], off[-1]), dtype=np.complex128)
    for (i, j), blk in bm.M.items():
        D[off[i]:off[i + 1], off[j]:off[j + 1]] = blk
    return D


def test_permuted_matrix_is_P_M_Pt():
    # test_matinvertndiag_ddrgf.jl:84-104 with ragged block sizes; blocks are
    # host arrays here: the permuted matrix only rearranges references
    rng = np.random.default_rng(4)
    sizes = list(rng.integers(2, 6, size=22))
    M = negf.BlockMatrix(sizes)
    for (i, j) in M.pattern("out"):
        M.M[(i, j)] = rng.standard_normal((sizes[i], sizes[j])) + 1j * rng.standard_normal((sizes[i], sizes[j]))
    perm_inv, _ = negf.bndiag_of_inv_ddrgf_create_permutation_vector(M, 4)
    perm = negf.bndiag_of_inv_ddrgf_transpose_permutation_vector(perm_inv)
    Mhat = negf.bndiag_of_inv_ddrgf_create_permuted_matrix(M, perm)
    for (i, j), blk in M.M.items():
        assert Mhat.M[(perm[i], perm[j])] is blk  # references, not copies
    # element permutation of the layers -> P M P^T
    off = M.offsets()
    idx = np.concatenate([np.arange(off[p], off[p + 1]) for p in perm_inv])
    D = _dense(M)
    assert np.array_equal(_dense(Mhat), D[np.ix_(idx, idx)])


def test_cost_model_pieces_match_oracle():
    for L in range(1, 9):
        for full in (False, True):
            if full and L > 4:
                with pytest.raises(negf.NegfError):
                    negf.cost_rgf(L, 2.0, 1.5, full)
                continue
            assert negf.cost_rgf(L, 2.0, 1.5, full) == o_dd.cost_rgf(L, 2.0, 1.5, full)
    for nr in (1, 2, 5, 13, 64):
        for thr in (1, 3, 8, 100):
            assert negf.bndiag_of_inv_ddrgf_check_nr_threads(thr, nr) == o_dd.check_nr_threads(thr, nr)
            for d1 in (1, 2, 3, 4):
                t = o_dd.check_nr_threads(thr, nr)[0]
                assert negf.cost_ddrgf(0.7, 2.5, nr, t, d1) == o_dd.cost_ddrgf(0.7, 2.5, nr, t, d1)


def test_bm_reference_and_build_M_from_HS():
    import scipy.sparse as sp
    rng = np.random.default_rng(1)
    big = {(i, j): rng.standard_normal((3, 3)) for i in range(8) for j in range(8)}
    M = negf.BlockMatrix([3] * 4, ndiag={"in": 3, "out": 3})
    negf.bm_reference_(M, big, 2, 2)
    for (i, j) in M.pattern("out"):
        assert M.M[(i, j)] is big[(i + 2, j + 2)]
    H = sp.random(30, 30, density=0.2, random_state=2, dtype=np.complex128)
    S = sp.identity(30, dtype=np.complex128, format="csc") + 0.1 * sp.random(30, 30, density=0.1, random_state=3)
    Se = sp.random(30, 30, density=0.05, random_state=4, dtype=np.complex128)
    Mm = negf.build_M_from_HS(H, S, Se, 0.37)
    assert np.allclose(Mm.toarray(), 0.37 * S.toarray() - H.toarray() - Se.toarray(), rtol=0, atol=0)


def test_sparse_permutator_matches_permuted_matrix():
    """The reference's DDRGF test compares P (M P^T) with the permuted block
    matrix (test_matinvertndiag_ddrgf.jl:84-110); the same check here."""
    rng = np.random.default_rng(4)
    sizes = [3, 5, 2, 4, 3, 6, 2, 5, 4, 3, 2, 4, 5, 3, 2, 4, 3, 5, 2, 4]
    M = negf.BlockMatrix(sizes, ndiag={"in": 3, "out": 3})
    for (i, j) in M.pattern("out"):
        M.M[(i, j)] = rng.standard_normal((sizes[i], sizes[j])) + 1j * rng.standard_normal((sizes[i], sizes[j]))
    perm_inv, _ = negf.bndiag_of_inv_ddrgf_create_permutation_vector(M, 4)
    perm = negf.bndiag_of_inv_ddrgf_transpose_permutation_vector(perm_inv)
    P = negf.bndiag_of_inv_ddrgf_create_sparse_permutator(perm, sizes)
    n = sum(sizes)
    assert P.shape == (n, n) and P.nnz == n
    assert np.array_equal((P @ P.T).toarray(), np.eye(n))
    D = _dense(M)
    Mhat = negf.bndiag_of_inv_ddrgf_create_permuted_matrix(M, perm)
    assert np.array_equal((P @ (sp.csc_matrix(D) @ P.T)).toarray(), _dense(Mhat))


def test_ddrgf_memory_estimate():
    # RGF buffers (1 block diagonal, 3 tridiagonal) + DDRGF's (1, 2); the
    # reference's 80 % comparison is disabled, so nothing raises
    for npl, b in ((16, 64), (64, 512), (4096, 1024)):
        mb = negf.check_if_enough_mem_ddrgf(npl, b)
        exp = negf.required_mem_non_symm(npl, 8, 1, 3, b) + negf.required_mem_non_symm(npl, 8, 1, 2, b)
        assert mb == exp > 0


def _pattern(keys, size=4):
    return {k: negf.Block(row=size + k[0], col=size + k[1]) for k in keys}


def test_block_index_helpers():
    """get_rc_index / get_rc_index_at(!) / get_row_index_at / get_col_index_at
    / get_colSizes / get_blockSizes (block.jl:348-501) on a selected-inverse
    pattern, 0-based, with the reference's inclusive range ends."""
    keys = [(0, 0), (0, 1), (1, 0), (1, 1), (1, 2), (2, 1), (2, 2), (2, 3), (3, 2), (3, 3), (0, 3)]
    A = _pattern(keys)
    rows, cols = negf.get_rc_index(A)
    assert list(zip(rows, cols)) == sorted(keys)
    assert negf.get_rc_index(A, 2, 2) == ([0, 0, 1, 1], [0, 1, 0, 1])
    buf = [99]
    negf.get_rc_index_at_(buf, A, 1, 2, 0, 3, True)
    assert buf == [1, 1, 1, 2, 2, 2]
    assert negf.get_rc_index_at(A, 1, 2, 0, 3, False) == [0, 1, 2, 1, 2, 3]
    # one assigned block per row / column of the range
    assert negf.get_row_index_at(A, 0, 3, 3, 3) == [0, 2, 3]
    assert negf.get_col_index_at(A, 3, 3, 0, 3) == [2, 3]
    with pytest.raises(IndexError):
        negf.get_row_index_at(A, 0, 1, 0, 3)  # five blocks, two rows: the reference's BoundsError
    assert negf.get_colSizes(A) == [4, 5, 6, 7]
    assert negf.get_blockSizes(A) == ([4, 5, 6, 7], [4, 5, 6, 7])
    assert negf.get_blockSizes(A, 2) == ([4, 5], [4, 5])


def test_bm_equal():
    """bm_equal (block.jl:223-243): same assigned blocks, equal contents."""
    rng = np.random.default_rng(2)
    keys = [(0, 0), (0, 1), (1, 0), (1, 1)]
    blocks = {k: rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3)) for k in keys}

    def make(src):
        out = {}
        for k, v in src.items():
            b = negf.Block(row=3, col=3)
            b.Full = v.copy()  # host blocks: the comparison needs no device
            out[k] = b
        return out

    A, B = make(blocks), make(blocks)
    assert negf.bm_equal(A, B)
    B[(0, 1)].Full[2, 2] += 1e-14
    assert not negf.bm_equal(A, B)
    C = make({k: v for k, v in blocks.items() if k != (1, 0)})
    assert not negf.bm_equal(A, C)
    D = make(blocks)
    D[(1, 1)].Full = D[(1, 1)].Full[:2, :2]
    assert not negf.bm_equal(A, D)
