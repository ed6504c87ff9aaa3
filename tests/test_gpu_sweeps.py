"""GPU parity of general RGF, the fused variant, the selected inverse, DDRGF,
the LU backend primitives and the reference's C entry point.

Tolerances follow the reference tests: 1e-12 for general RGF / fused
(test_matinvertndiag_general_rgf*.jl, roundoffs[ComplexF64]*1e3), 2.5e-10 for
DDRGF vs sequential RGF (test_matinvertndiag_ddrgf.jl:16), 1e-13 absolute for
the selected inverse (test_selected_inverse.jl:51) and 1e-15-scale relative
for the block LU (:20-21, relaxed to 1e-14 for GPU summation order).
"""

import ctypes

import numpy as np
import pytest

from conftest import kappa_tol, rel_fro
from oracle import rgf as o_rgf, general_rgf as o_grgf, selected_inverse as o_si, ddrgf as o_dd
from oracle import direct as o_direct
from oracle.blockmatrix import bm_convert_dense, band_of_dense, bm_fuse_to_tridiagonal as o_fuse
from oracle.generators import bm_create_synthetic_random, set_sparse_block, full_of_blocks

pytestmark = pytest.mark.gpu


def _to_gpu_bm(negf, bm):
    out = negf.BlockMatrix(bm.blockSizes, None, bm.ndiag, False, bm.isHermitian)
    for k, v in bm.M.items():
        out.M[k] = negf.to_device(v)
    return out


@pytest.mark.parametrize("npl,b,nd", [(10, 32, 5), (7, 20, 7), (6, 40, 3), (3, 16, 5), (1, 8, 5)])
def test_general_rgf(negf, npl, b, nd):
    M = bm_create_synthetic_random(npl, b, seed=npl + b + nd, ndiag=nd)
    ref = bm_convert_dense(o_grgf.bndiag_of_inv_general_rgf(M))
    dM = _to_gpu_bm(negf, M)
    before = {k: negf.to_host(v).copy() for k, v in dM.M.items()}
    out = negf.BlockMatrix(M.blockSizes)
    negf.bndiag_of_inv_general_rgf_(out, dM, negf.allocate_aux_data_general_RGF(dM))
    G = negf.bm_to_dense(out)
    # the reference's 1e-12 (roundoffs[ComplexF64] * 1e3), widened to 2 u kappa for
    # the worse-conditioned draws of the uniform-[0,1) generator
    D = bm_convert_dense(M)
    tol = kappa_tol(np.linalg.cond(D))
    assert rel_fro(G, ref) < tol
    exact = band_of_dense(np.linalg.inv(D), M.blockSizes, {"in": nd, "out": nd})
    assert rel_fro(G, exact) < tol
    for k, v in dM.M.items():  # input left unchanged
        assert np.array_equal(negf.to_host(v), before[k])


def test_general_rgf_vs_fused(negf):
    # test_matinvertndiag_general_rgf_fused.jl: general n-diagonal RGF vs fuse + RGF
    M = bm_create_synthetic_random(10, 32, seed=77, ndiag=5)
    dM = _to_gpu_bm(negf, M)
    gen = negf.BlockMatrix(M.blockSizes)
    negf.bndiag_of_inv_general_rgf_(gen, dM)
    fused = negf.bm_fuse_to_tridiagonal(dM)
    o_fused = o_fuse(M)
    assert rel_fro(negf.bm_to_dense(fused), bm_convert_dense(o_fused)) == 0.0
    fout = negf.BlockMatrix(fused.blockSizes)
    negf.bndiag_of_inv_rgf_local_(fout, fused)
    aligned = band_of_dense(negf.bm_to_dense(fout), M.blockSizes, {"in": 5, "out": 5})
    assert rel_fro(negf.bm_to_dense(gen), aligned) < kappa_tol(np.linalg.cond(bm_convert_dense(M)))


RIND = [1, 1, 1, 2, 3, 3, 3, 4, 5]
CIND = [1, 3, 5, 2, 3, 4, 5, 4, 5]


def _gpu_blocks(negf, A):
    return {k: negf.Block(negf.to_device(v)) for k, v in A.items()}


@pytest.mark.parametrize("bs", [100, 1, 33])
def test_block_factorization(negf, bs):
    A = set_sparse_block([bs] * 5, RIND, CIND, True, seed=bs)
    F_ref = o_si.block_factorization(A, 5)
    F = negf.Block_factorization(_gpu_blocks(negf, A))
    Fm = negf.full(F, 5)
    assert rel_fro(Fm, full_of_blocks(F_ref, [bs] * 5)) < 1e-14
    # test_selected_inverse.jl:17-21
    T = full_of_blocks(A, [bs] * 5)
    n = 5 * bs
    LU = (np.tril(Fm, -1) + np.eye(n)) @ np.triu(Fm)
    assert rel_fro(LU, T) < 1e-14
    import scipy.linalg as sl
    P, L, U = sl.lu(T)
    if np.allclose(P, np.eye(n)):
        assert rel_fro(Fm, np.tril(L, -1) + U) < 1e-14


@pytest.mark.parametrize("bs", [1, 100, 24])
def test_block_inverse(negf, bs):
    A = set_sparse_block([bs] * 5, RIND, CIND, True, seed=10 + bs)
    T = full_of_blocks(A, [bs] * 5)
    Z_ref = o_si.block_inverse(o_si.block_factorization(A, 5), 5)
    Z = negf.Block_inverse(negf.Block_factorization(_gpu_blocks(negf, A)))
    invT = np.linalg.inv(T)
    for (i, j), blk in Z.items():
        z = negf.to_host(blk.Full)
        assert np.allclose(z, invT[i * bs:(i + 1) * bs, j * bs:(j + 1) * bs], atol=1e-13, rtol=0)
        assert np.allclose(z, Z_ref[(i, j)], atol=1e-13, rtol=0)
    # diag(A * si(A)) = 1 (test_selected_inverse.jl:38-42) on the full inverse
    full = negf.full(Z, 5)
    mask = np.zeros_like(T, dtype=bool)
    for (i, j) in Z:
        mask[i * bs:(i + 1) * bs, j * bs:(j + 1) * bs] = True
    assert np.all(np.abs(full[mask] - invT[mask]) < 1e-13)


@pytest.mark.parametrize("n", [5, 64, 96, 97, 200, 513])
def test_getrf_trsm_getri(negf, n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    import scipy.linalg.lapack as la
    lu_ref, piv_ref, info = la.zgetrf(A)
    dA = negf.to_device(A)
    lib = negf.load()
    import torch
    piv = torch.zeros(n, dtype=torch.int32, device="cuda")
    from libnegf_b200._lib import int_array, ptr_array, check
    infos = (ctypes.c_int32 * 1)()
    check(lib.negf_zgetrf_batched(1, int_array([n]), ptr_array([dA.data_ptr()]), int_array([n]),
                                  ptr_array([piv.data_ptr()]), infos, None))
    assert np.array_equal(piv.cpu().numpy() - 1, piv_ref)
    assert rel_fro(negf.to_host(dA), lu_ref) < 1e-13
    # trsm with the factors: the four forms used by selected_inverse.jl
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    U = np.triu(lu_ref)
    L = np.tril(lu_ref, -1) + np.eye(n)
    cases = [("R", "U", "N", 1.0, B @ np.linalg.inv(U)), ("L", "L", "U", 1.0, np.linalg.solve(L, B)),
             ("L", "U", "N", -1.0, -np.linalg.solve(U, B)), ("R", "L", "U", -1.0, -B @ np.linalg.inv(L))]
    for side, uplo, diag, a, ref in cases:
        alpha = (ctypes.c_double * 2)(a, 0.0)
        dB = negf.to_device(B)
        check(lib.negf_ztrsm_batched(side.encode(), uplo.encode(), b"N", diag.encode(), alpha, 1, int_array([n]),
                                     int_array([n]), ptr_array([dA.data_ptr()]), int_array([n]),
                                     ptr_array([dB.data_ptr()]), int_array([n]), None))
        assert rel_fro(negf.to_host(dB), ref) < 1e-11
    check(lib.negf_zgetri_nopiv_batched(1, int_array([n]), ptr_array([dA.data_ptr()]), int_array([n]), None))
    assert rel_fro(negf.to_host(dA), np.linalg.inv(U) @ np.linalg.inv(L)) < 1e-11


@pytest.mark.parametrize("npl,b,d1", [(32, 16, 6), (128, 24, 15), (20, 40, 4), (18, 8, 3), (8, 30, 1)])
def test_ddrgf_vs_rgf(negf, npl, b, d1):
    M = bm_create_synthetic_random(npl, b, seed=npl * 3 + d1)
    seq = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(M))
    o_par, _ = o_dd.bndiag_of_inv_ddrgf(M, d1)
    assert rel_fro(bm_convert_dense(o_par), seq) < 2.5e-10
    dM = _to_gpu_bm(negf, M)
    aux = negf.allocate_aux_data_DDRGF(dM, blockSizeD1=d1)
    assert aux[0].nrTasks == o_dd.get_nr_tasks(npl, d1)[0]
    negf.bndiag_of_inv_ddrgf_(dM, aux)
    G = negf.bm_to_dense(aux[0].buffMout)
    assert rel_fro(G, seq) < 2.5e-10
    assert rel_fro(G, bm_convert_dense(o_par)) < 2.5e-10


def test_ddrgf_auto_partition(negf):
    M = bm_create_synthetic_random(40, 16, seed=9)
    dM = _to_gpu_bm(negf, M)
    aux = negf.allocate_aux_data_DDRGF(dM)
    negf.bndiag_of_inv_ddrgf_(dM, aux)
    seq = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(M))
    assert rel_fro(negf.bm_to_dense(aux[0].buffMout), seq) < 2.5e-10


@pytest.mark.parametrize("npl,b,d1s", [(128, 16, [4, 3]), (64, 24, [3, 1, 1]), (40, 12, [3, 1, 2]),
                                       (128, 8, [7, 7]), (200, 8, None)])
def test_ddrgf_multilevel_vs_rgf(negf, npl, b, d1s):
    # the recursion of bndiag_of_inv_ddrgf! through _inv_Schur_compl!
    # (matinvertndiag_ddrgf_core.jl:656-680); None = the GPU cost model's levels
    M = bm_create_synthetic_random(npl, b, seed=npl * 7 + b)
    seq = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(M))
    dM = _to_gpu_bm(negf, M)
    aux = negf.allocate_aux_data_DDRGF(dM, blockSizeD1=d1s)
    used = [a.blockSizeD1 for a in aux]
    if d1s is not None:
        assert used == d1s
    else:
        assert len(used) >= 2, used
    n = npl
    for a in aux:  # task counts chain through the levels as the oracle's partition
        assert a.nrTasks == o_dd.get_nr_tasks(n, a.blockSizeD1)[0]
        n = a.nrTasks
    negf.bndiag_of_inv_ddrgf_(dM, aux)
    G = negf.bm_to_dense(aux[0].buffMout)
    assert rel_fro(G, seq) < 2.5e-10
    o_par, _ = o_dd.bndiag_of_inv_ddrgf(M, used)
    assert rel_fro(G, bm_convert_dense(o_par)) < 2.5e-10


def test_ddrgf_reference_cost_model(negf):
    # test_matinvertndiag_ddrgf.jl:13-14, :86-158: npl = 128, b = 64, levels from
    # allocate_aux_data_DDRGF's probes + opt_params (here the probes time the
    # library's kernels), DDRGF vs sequential RGF at 2.5e-10
    M = bm_create_synthetic_random(128, 64, seed=1234)
    seq = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(M))
    dM = _to_gpu_bm(negf, M)
    rlu, rml = negf.get_rLU(dM), negf.get_rMLDIV(dM)
    assert rlu[0] > 0 and rml[0] > 0
    aux = negf.allocate_aux_data_DDRGF(dM, costModel="reference", nrThreads=8)
    assert 1 <= len(aux) <= 6 and all(1 <= a.blockSizeD1 <= 4 for a in aux)
    negf.bndiag_of_inv_ddrgf_(dM, aux)
    assert rel_fro(negf.bm_to_dense(aux[0].buffMout), seq) < 2.5e-10


def test_ddrgf_levels_batched_uneven_and_errors(negf):
    # two systems of 48 layers with different block sizes in one call, upper /
    # lower outputs not requested (NULL); then an impossible coarse partition
    from libnegf_b200._lib import NegfError, check, int_array, ptr_array
    lib = negf.load()
    npl, d1s = 48, [3, 2]
    mats = [bm_create_synthetic_random(npl, 10, seed=3), bm_create_synthetic_random(npl, 17, seed=4)]
    keep, sizes, Md, Mu, Ml, Gd, outs = [], [], [], [], [], [], []
    for M in mats:
        sizes += M.blockSizes
        for i in range(npl):
            keep.append(negf.to_device(M.M[(i, i)])); Md.append(keep[-1].data_ptr())
        for i in range(npl - 1):
            keep.append(negf.to_device(M.M[(i, i + 1)])); Mu.append(keep[-1].data_ptr())
            keep.append(negf.to_device(M.M[(i + 1, i)])); Ml.append(keep[-1].data_ptr())
        o = [negf.dzeros(b, b) for b in M.blockSizes]
        outs.append(o)
        Gd += [t.data_ptr() for t in o]
    check(lib.negf_ddrgf_levels(2, npl, int_array(sizes), ptr_array(Md), ptr_array(Mu), ptr_array(Ml), len(d1s),
                                int_array(d1s), ptr_array(Gd), None, None, None))
    for M, o in zip(mats, outs):
        ref, _ = o_dd.bndiag_of_inv_ddrgf(M, d1s)
        for i in range(npl):
            assert rel_fro(negf.to_host(o[i]), ref.M[(i, i)]) < 2.5e-10
    # 48 layers, D1 = 3: 12 separators; D1 = 2 on 12 layers: 4 tasks; D1 = 2 on 4
    # layers is impossible (get_nr_tasks = -1): rejected before any launch
    assert o_dd.get_nr_tasks(4, 2)[0] == -1
    bad = [3, 2, 2]
    with pytest.raises(NegfError):
        check(lib.negf_ddrgf_levels(2, npl, int_array(sizes), ptr_array(Md), ptr_array(Mu), ptr_array(Ml), 3,
                                    int_array(bad), ptr_array(Gd), None, None, None))


def test_run_bndiag_wrapper(negf):
    # the reference C example (src/c_interface/libnegf_c_example.c) builds a
    # random block tridiagonal CSC matrix and calls run_bndiag_wrapper
    import scipy.sparse as sp
    from libnegf_b200._lib import int_array
    npl, b = 12, 16
    M = bm_create_synthetic_random(npl, b, seed=123, uniform=True)
    D = bm_convert_dense(M)
    csc = sp.csc_matrix(D)
    n = D.shape[0]
    colptr = np.ascontiguousarray(csc.indptr, dtype=np.int32)
    rowval = np.ascontiguousarray(csc.indices, dtype=np.int32)
    nz = np.ascontiguousarray(csc.data, dtype=np.complex128)
    keys = (ctypes.c_char_p * 2)(b"in", b"out")
    lib = negf.load()
    res = lib.run_bndiag_wrapper(n, n, csc.nnz, colptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                 rowval.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nz.ctypes.data, npl,
                                 int_array([b] * npl), 2, keys, int_array([3, 3]), 0)
    assert res.m == n and res.nnz > 0
    cp = np.ctypeslib.as_array(res.colptr, shape=(n + 1,)).copy()
    rv = np.ctypeslib.as_array(res.rowval, shape=(res.nnz,)).copy()
    vals = np.ctypeslib.as_array(ctypes.cast(res.nzval, ctypes.POINTER(ctypes.c_double)), shape=(2 * res.nnz,)).copy()
    out = sp.csc_matrix((vals[0::2] + 1j * vals[1::2], rv, cp), shape=(n, n)).toarray()
    libc = ctypes.CDLL(None)
    for p in (res.colptr, res.rowval, res.nzval):
        libc.free(ctypes.cast(p, ctypes.c_void_p))
    ref = band_of_dense(np.linalg.inv(D), M.blockSizes, {"in": 3, "out": 3})
    assert rel_fro(out, ref) < 2.5e-10


def _call_wrapper(negf, D, npl, b, out_nd, hermitian):
    import scipy.sparse as sp
    from libnegf_b200._lib import int_array
    csc = sp.csc_matrix(D)
    csc.sort_indices()
    n = D.shape[0]
    colptr = np.ascontiguousarray(csc.indptr, dtype=np.int32)
    rowval = np.ascontiguousarray(csc.indices, dtype=np.int32)
    nz = np.ascontiguousarray(csc.data, dtype=np.complex128)
    keys = (ctypes.c_char_p * 2)(b"in", b"out")
    lib = negf.load()
    sizes = b if isinstance(b, list) else [b] * npl
    res = lib.run_bndiag_wrapper(n, n, csc.nnz, colptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                 rowval.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nz.ctypes.data, npl,
                                 int_array(sizes), 2, keys, int_array([3, out_nd]), int(hermitian))
    assert res.m == n and res.nnz > 0
    cp = np.ctypeslib.as_array(res.colptr, shape=(n + 1,)).copy()
    rv = np.ctypeslib.as_array(res.rowval, shape=(res.nnz,)).copy()
    vals = np.ctypeslib.as_array(ctypes.cast(res.nzval, ctypes.POINTER(ctypes.c_double)), shape=(2 * res.nnz,)).copy()
    libc = ctypes.CDLL(None)
    for p in (res.colptr, res.rowval, res.nzval):
        libc.free(ctypes.cast(p, ctypes.c_void_p))
    # every column's rows are sorted and inside the matrix
    for c in range(n):
        r = rv[cp[c]:cp[c + 1]]
        assert np.all(np.diff(r) > 0) and (r.size == 0 or (r[0] >= 0 and r[-1] < n))
    return sp.csc_matrix((vals[0::2] + 1j * vals[1::2], rv, cp), shape=(n, n)).toarray()


def test_run_bndiag_wrapper_hermitian_ragged(negf):
    from oracle import physics as o_phys
    sizes = [24, 40, 16, 32, 24]
    s = o_phys.physics_system(len(sizes), 0, seed=31, block_sizes=sizes)
    n = sum(sizes)
    off = np.cumsum([0] + sizes)
    H = np.zeros((n, n), dtype=np.complex128)
    for i, h in enumerate(s.Hd):
        H[off[i]:off[i + 1], off[i]:off[i + 1]] = h
    for i, h in enumerate(s.Hu):
        H[off[i]:off[i + 1], off[i + 1]:off[i + 2]] = h
        H[off[i + 1]:off[i + 2], off[i]:off[i + 1]] = h.conj().T
    D = 0.3 * np.eye(n) - H  # Hermitian, M = E - H at a real energy
    D[np.abs(D) < 1e-3] = 0.0
    # the full matrix is passed; with is_hermitian only its diagonal and upper
    # blocks are read (src/c_interface/libnegf_c_interface.jl:115-121)
    out = _call_wrapper(negf, D, len(sizes), sizes, 3, True)
    ref = band_of_dense(np.linalg.inv(D), sizes, {"in": 3, "out": 3})
    assert rel_fro(out, ref) < 2.5e-10 * max(1.0, np.linalg.cond(D) / 1e4)


def test_run_bndiag_wrapper_wide_out_band(negf):
    # "out" = 5: the tridiagonal of the inverse plus the input's blocks at
    # distance 2 (absent in a tridiagonal input), through the device lookup
    npl, b = 8, 24
    M = bm_create_synthetic_random(npl, b, seed=77, uniform=True)
    D = bm_convert_dense(M)
    out = _call_wrapper(negf, D, npl, b, 5, False)
    ref = band_of_dense(np.linalg.inv(D), M.blockSizes, {"in": 3, "out": 3})
    assert rel_fro(out, ref) < 2.5e-10 * max(1.0, np.linalg.cond(D) / 1e4)


def _direct_case(negf, M, sizes, nd_out):
    import scipy.sparse as sp
    A = sp.csc_matrix(M)
    R = negf.bndiag_of_inv_direct(A, sizes, {"in": 3, "out": nd_out})
    ref, inv = o_direct.bndiag_of_inv_direct(A, sizes, {"in": 3, "out": nd_out})
    return R, ref, inv


@pytest.mark.parametrize("npl,b,nd_out", [(12, 32, 3), (6, 50, 5), (10, 128, 3), (3, 7, 3), (1, 40, 3)])
def test_bndiag_of_inv_direct(negf, npl, b, nd_out):
    # test_matinvertndiag_direct.jl:34-47: relErr (2-norm) of the direct band
    # against the reference band < roundoff * cond * 10; n = 1280 (10 x 128)
    # takes the block-elimination form, the others one Gauss-Jordan inverse
    Mb = bm_create_synthetic_random(npl, b, seed=npl * 11 + b)
    D = bm_convert_dense(Mb)
    R, ref, inv = _direct_case(negf, D, Mb.blockSizes, nd_out)
    G = R.toarray()
    cond = np.linalg.cond(D)
    assert np.linalg.norm(G - ref, 2) / np.linalg.norm(ref, 2) < 1e-15 * cond * 10
    # and against RGF's tridiagonal of the inverse (an independent method)
    if nd_out == 3 and npl > 1:
        seq = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(Mb))
        assert rel_fro(G, seq) < kappa_tol(cond)
    # stored pattern: the out band of the inverse (no exact zeros there)
    off = np.concatenate([[0], np.cumsum(Mb.blockSizes)])
    w = (nd_out - 1) // 2
    mask = np.zeros_like(D, dtype=bool)
    for i in range(npl):
        for j in range(max(0, i - w), min(npl, i + w + 1)):
            mask[off[i]:off[i + 1], off[j]:off[j + 1]] = True
    assert R.nnz == int(mask.sum())
    assert np.all(R.toarray()[~mask] == 0)


def test_bndiag_of_inv_direct_keeps_entries_outside_the_band(negf):
    # a pentadiagonal input with a tridiagonal output: the reference writes the
    # tridiagonal of the inverse into M, whose other stored entries stay
    import scipy.sparse as sp
    Mb = bm_create_synthetic_random(8, 24, seed=21, ndiag=5)
    D = bm_convert_dense(Mb)
    A = sp.csc_matrix(D)
    R, ref, inv = _direct_case(negf, D, Mb.blockSizes, 3)
    G = R.toarray()
    off = np.concatenate([[0], np.cumsum(Mb.blockSizes)])
    band = np.zeros_like(D, dtype=bool)
    for i in range(8):
        for j in range(max(0, i - 1), min(8, i + 2)):
            band[off[i]:off[i + 1], off[j]:off[j + 1]] = True
    assert np.array_equal(G[~band], D[~band])  # bit-exact copies of M
    assert rel_fro(G[band], inv[band]) < 1e-12
    # in place on a scipy matrix
    negf.bndiag_of_inv_direct_(A, Mb.blockSizes, {"in": 5, "out": 3})
    assert np.array_equal(A.toarray(), G)


def test_bndiag_of_inv_direct_rejects_bad_input(negf):
    import scipy.sparse as sp
    from libnegf_b200 import NegfError
    D = np.eye(8, dtype=np.complex128)
    with pytest.raises(NegfError):
        negf.bndiag_of_inv_direct(sp.csc_matrix(D), [4, 3], {"out": 3})  # sizes do not add up
    with pytest.raises(NegfError):
        negf.bndiag_of_inv_direct(sp.csc_matrix(D), [4, 4], {"out": 4})  # even band


def test_backend_getrf_trsm_getri_mirror(negf):
    # be_getrf! / be_trsm! / be_getri! (backend_cpu.jl:229-265) through the mirror
    import scipy.linalg as sla
    rng = np.random.default_rng(12)
    n = 70
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 12 * np.eye(n)
    lu_ref, piv_ref = sla.lu_factor(A)
    dA = negf.to_device(A)
    assert negf.be_getrf_(dA) == 0
    assert rel_fro(negf.to_host(dA), lu_ref) < 1e-13
    assert np.array_equal(piv_ref, np.arange(n))  # diagonally dominant: no interchanges
    B = rng.standard_normal((n, 30)) + 1j * rng.standard_normal((n, 30))
    dB = negf.to_device(B)
    negf.be_trsm_("L", "L", "N", "U", 1.0, dA, dB)
    L = np.tril(lu_ref, -1) + np.eye(n)
    assert rel_fro(negf.to_host(dB), np.linalg.solve(L, B)) < 1e-12
    negf.be_getri_(dA)
    assert rel_fro(negf.to_host(dA), np.linalg.inv(A)) < 1e-12


@pytest.mark.parametrize("npl,b,d1", [(24, 12, 4), (19, 9, 3)])
def test_ddrgf_error_inv_of_T11(negf, npl, b, d1):
    # ddrgf_utils.jl:776-824: the interior domains' inverses reproduce the identity
    M = bm_create_synthetic_random(npl, b, seed=npl + d1)
    dM = _to_gpu_bm(negf, M)
    aux = negf.allocate_aux_data_DDRGF(dM, blockSizeD1=d1)
    a = aux[0]
    assert a.permVecInv == o_dd.partition(npl, d1)[2]
    err = negf.bndiag_of_inv_ddrgf_error_inv_of_T11(dM, a.buffMout, a)
    assert 0.0 < err < 1e-12
    single = negf.allocate_aux_data_DDRGF_single_level(dM, d1)
    assert single.nrTasks == a.nrTasks and single.permVec == a.permVec
