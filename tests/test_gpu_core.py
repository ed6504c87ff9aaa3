"""GPU parity of the core kernels and sweeps against the CPU oracle.

Tolerances: 1e-12 relative Frobenius for FP64 sweeps (the reference's
ComplexF64 test tolerance roundoffs[ComplexF64] * 1e3,
test/common_to_test.jl:25-27 and test_keldyshndiag.jl:18), 1e-13 for single
products.
"""

import numpy as np
import pytest

from conftest import kappa_tol, rel_fro
from oracle import rgf as o_rgf, keldysh as o_keldysh, physics as o_phys
from oracle.blockmatrix import bm_convert_dense, band_of_dense
from oracle.generators import bm_create_synthetic_random, hermitian_random_like

pytestmark = pytest.mark.gpu

TOL = 1e-12


def tol_ref(M):
    """The reference's ComplexF64 tolerance (1e-12), widened to 2 u kappa(M)
    for the worse-conditioned stress matrices."""
    return kappa_tol(np.linalg.cond(bm_convert_dense(M)), TOL)


def _rand(rng, m, n):
    return rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))


@pytest.mark.parametrize("ops", ["NN", "NC", "CN", "CC", "TN", "NT"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (37, 45, 29), (130, 70, 257), (1, 1, 1), (256, 256, 256)])
def test_zgemm_batched(negf, ops, shape):
    rng = np.random.default_rng(hash((ops, shape)) % 2 ** 32)
    m, n, k = shape
    tA, tB = ops
    A = _rand(rng, *((m, k) if tA == "N" else (k, m)))
    B = _rand(rng, *((k, n) if tB == "N" else (n, k)))
    C = _rand(rng, m, n)
    op = {"N": lambda x: x, "T": lambda x: x.T, "C": lambda x: x.conj().T}
    alpha, beta = 0.7 - 0.2j, -1.3 + 0.5j
    ref = alpha * op[tA](A) @ op[tB](B) + beta * C
    dA, dB, dC = negf.to_device(A), negf.to_device(B), negf.to_device(C)
    negf.be_gemm_(tA, tB, alpha, dA, dB, beta, dC)
    assert rel_fro(negf.to_host(dC), ref) < 1e-13


def test_zgemm_batched_ragged(negf):
    rng = np.random.default_rng(5)
    items, refs = [], []
    for (m, n, k) in [(60, 68, 61), (64, 64, 64), (3, 100, 7), (200, 5, 90)]:
        A, B, C = _rand(rng, m, k), _rand(rng, k, n), _rand(rng, m, n)
        refs.append(-A @ B + C)
        dC = negf.to_device(C)
        items.append((-1.0, negf.to_device(A), negf.to_device(B), 1.0, dC))
    negf.be_gemm_batched_("N", "N", items)
    for it, ref in zip(items, refs):
        assert rel_fro(negf.to_host(it[4]), ref) < 1e-13


@pytest.mark.parametrize("n", [1, 5, 32, 64, 100, 112, 113, 128, 256, 300, 512])
def test_zinv_batched(negf, n):
    rng = np.random.default_rng(n)
    As = [_rand(rng, n, n) for _ in range(3)]
    dA = [negf.to_device(a) for a in As]
    dO = [negf.dzeros(n, n) for _ in As]
    negf.be_inv_batched_(dA, dO)
    for a, o, da in zip(As, dO, dA):
        ref = np.linalg.inv(a)
        assert rel_fro(negf.to_host(o), ref) < 1e-12 * max(1.0, np.linalg.cond(a) / 1e2)
        assert np.array_equal(negf.to_host(da), a)  # input untouched


def test_zinv_singular(negf):
    a = np.zeros((8, 8), dtype=complex)
    a[:4, :4] = np.eye(4)
    with pytest.raises(negf.SingularError):
        negf.be_inv(negf.to_device(a))


def _to_gpu_bm(negf, bm):
    out = negf.BlockMatrix(bm.blockSizes, None, bm.ndiag, False, bm.isHermitian)
    for k, v in bm.M.items():
        out.M[k] = negf.to_device(v)
    return out


def _gpu_bm_dense(negf, bm):
    return negf.bm_to_dense(bm)


@pytest.mark.parametrize("npl,b,uniform", [(10, 32, False), (16, 64, True), (5, 130, False), (1, 40, True),
                                           (2, 20, False)])
def test_rgf_vs_oracle(negf, npl, b, uniform):
    M = bm_create_synthetic_random(npl, b, seed=npl * 7 + b, uniform=uniform)
    G_ref = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(M))
    dM = _to_gpu_bm(negf, M)
    dOut = negf.bm_copy(dM)
    negf.bndiag_of_inv_rgf_local_(dOut, dM, negf.allocate_aux_data_RGF(dM))
    G = _gpu_bm_dense(negf, dOut)
    tol = tol_ref(M)
    assert rel_fro(G, G_ref) < tol
    # and against the dense inverse (the reference test oracle)
    D = bm_convert_dense(M)
    assert rel_fro(G, band_of_dense(np.linalg.inv(D), M.blockSizes, {"in": 3, "out": 3})) < tol


def test_rgf_full_inverse(negf):
    M = bm_create_synthetic_random(6, 24, seed=3)
    dM = _to_gpu_bm(negf, M)
    dOut = negf.BlockMatrix(dM.blockSizes)
    negf.bndiag_of_inv_rgf_local_(dOut, dM, negf.allocate_aux_data_RGF(dM, buildFullInv=True))
    G = _gpu_bm_dense(negf, dOut)
    assert rel_fro(G, np.linalg.inv(bm_convert_dense(M))) < tol_ref(M)


def test_rgf_batched_systems(negf):
    Ms = [bm_create_synthetic_random(8, 48, seed=s, uniform=True) for s in range(4)]
    dMs = [_to_gpu_bm(negf, m) for m in Ms]
    outs = [negf.BlockMatrix(m.blockSizes) for m in dMs]
    negf.bndiag_of_inv_rgf_local_batched_(outs, dMs)
    for M, o in zip(Ms, outs):
        ref = bm_convert_dense(o_rgf.bndiag_of_inv_rgf_local(M))
        assert rel_fro(_gpu_bm_dense(negf, o), ref) < tol_ref(M)


@pytest.mark.parametrize("npl,b", [(10, 32), (4, 64), (2, 16), (3, 150)])
def test_keldysh_vs_oracle(negf, npl, b):
    M = bm_create_synthetic_random(npl, b, seed=100 + npl)
    S = hermitian_random_like(M, seed=200 + npl)
    ref = bm_convert_dense(o_keldysh.keldyshndiag(M, S))
    dM = _to_gpu_bm(negf, M)
    dS = _to_gpu_bm(negf, S)
    aux = negf.allocate_aux_data_Keldysh(dM, dS)
    negf.keldyshndiag_(dM, dS, aux)
    G = _gpu_bm_dense(negf, aux.buffS)
    tol = tol_ref(M)
    assert rel_fro(G, ref) < tol
    # dense check as in test_keldyshndiag.jl:80-95
    D = bm_convert_dense(M)
    Gr = np.linalg.inv(D)
    bf = Gr @ bm_convert_dense(S) @ Gr.conj().T
    assert rel_fro(G, band_of_dense(bf, M.blockSizes, {"in": 3, "out": 3}, True)) < tol


@pytest.mark.parametrize("npl,b,nE", [(6, 32, 5), (4, 100, 3), (1, 16, 2)])
def test_negf_device_solve(negf, npl, b, nE):
    sysm = o_phys.physics_system(npl, b, seed=11)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    Es = np.linspace(-0.9, 0.8, nE)
    gr, gl, t = dev.solve(Es, eta=sysm.eta)
    for e, E in enumerate(Es):
        r = o_phys.solve_energy(sysm, E)
        for i in range(npl):
            assert rel_fro(gr[e][i], r["GR"].M[(i, i)]) < TOL
            assert rel_fro(gl[e][i], 1j * r["Gn"].M[(i, i)]) < TOL
        assert abs(t[e] - r["T"]) <= 1e-10 * max(1.0, abs(r["T"]))


def test_negf_solver_chunked(negf):
    sysm = o_phys.physics_system(5, 40, seed=2)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    Es = np.linspace(-1, 1, 7)
    gr1, gl1, t1 = dev.solve(Es, eta=sysm.eta)
    gr2, gl2, t2 = dev.solve(Es, eta=sysm.eta, max_chunk=3)
    for e in range(len(Es)):
        for i in range(5):
            assert rel_fro(gr2[e][i], gr1[e][i]) < 1e-14
            assert rel_fro(gl2[e][i], gl1[e][i]) < 1e-14
    assert np.allclose(t1, t2, rtol=1e-13, atol=0)
