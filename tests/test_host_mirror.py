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
