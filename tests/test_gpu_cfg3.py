"""Batched selected inverse and DDRGF over energies, FP64 and mixed precision.

The configuration these cover: the selected inverse (tridiagonal blocks of
G^R(E) = M(E)^{-1}) of one device for many energies, by domain-decomposed RGF
(bndiag_of_inv_ddrgf!, src/matinvertndiag_ddrgf_core.jl:719-758, four
partitions) and by the block selected inverse (Block_factorization! +
Block_inverse!, src/selected_inverse.jl:9-206), every recursion step one
launch over all energies, with the block products in FP64 or on the INT8
tensor cores (mixed).

Bars: DDRGF (both precisions) against the oracle's DDRGF restatement with the
same levels. With eta = 1e-2 every interior domain is well conditioned and the
bar is the reference's DDRGF tolerance, 2.5e-10
(test_matinvertndiag_ddrgf.jl:245-293). With eta = 1e-6 the interior domains
are closed systems (no lead self-energy) whose inverses are ill-conditioned:
DDRGF itself -- the reference's algorithm, restated on the CPU -- departs from
sequential RGF by up to ~3e-8 at b = 512, and a relative perturbation of the
input at the unit roundoff moves it by as much. There the bar is 2.5e-10 plus
30x the larger of those two figures at the same energy (two backward-stable
executions of DDRGF -- LAPACK LU solves on the CPU, Gauss-Jordan inverses on
the GPU -- differ by up to ~10x that sensitivity). Sequential RGF on the same
device stays within 1e-11 of the oracle's. The selected inverse on the
NEGF generator (lu(NoPivot()) diagonal factorisations) against the oracle's
restatement with the same factorisation and the dense inverse at 1e-12 (FP64)
/ 1e-10 (mixed); the batched reference-API entry point against the oracle's
restatement of the reference (be_getrf! with discarded pivots) on the
reference test's diagonally dominant generator at 1e-13 absolute.
"""

import copy

import numpy as np
import pytest

from conftest import rel_fro
from oracle import ddrgf as o_ddrgf, physics as o_phys, rgf as o_rgf, selected_inverse as o_si
from oracle.blockmatrix import bm_convert_dense
from oracle.generators import set_sparse_block, full_of_blocks

pytestmark = pytest.mark.gpu


def _max_err(got, ref):
    return max(rel_fro(g, r) for g, r in zip(got, ref))


def _oracle_tri(sysm, E):
    M = sysm.M_of_E(E)
    G = o_rgf.bndiag_of_inv_rgf_local(M)
    n = sysm.npl
    return ([G.M[(i, i)] for i in range(n)], [G.M[(i, i + 1)] for i in range(n - 1)],
            [G.M[(i + 1, i)] for i in range(n - 1)])


def _perturbed(M, rng):
    """M with every stored block scaled entrywise by (1 + 2^-53 z), z complex normal."""
    P = copy.deepcopy(M)
    for k, v in P.M.items():
        P.M[k] = v * (1.0 + 2.0 ** -53 * (rng.standard_normal(v.shape) + 1j * rng.standard_normal(v.shape)))
    return P


def _tri_of(D, n):
    return ([D.M[(i, i)] for i in range(n)], [D.M[(i, i + 1)] for i in range(n - 1)],
            [D.M[(i + 1, i)] for i in range(n - 1)])


@pytest.mark.parametrize("npl,b,nE,levels,eta", [(16, 512, 4, [3], 1e-2), (16, 512, 4, [3], 1e-6),
                                                 (19, 64, 5, [4], 1e-6), (40, 32, 3, [3, 3], 1e-6)])
def test_device_ddrgf_fp64_and_mixed(negf, npl, b, nE, levels, eta):
    """DDRGF of the NEGF generator over energies; (16, 512, [3]) is the
    benchmark's b = 512 with four partitions (separators at layers 0, 4, 8, 12)."""
    sysm = o_phys.physics_system(npl, b, seed=31, eta=eta)
    Es = np.linspace(-0.7, 0.8, nE)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    f64 = dev.selected_inverse(Es, method="ddrgf", precision="fp64", eta=sysm.eta, levels=levels)
    mix = dev.selected_inverse(Es, method="ddrgf", precision="mixed", eta=sysm.eta, levels=levels)
    rgf = dev.selected_inverse(Es, method="rgf", precision="fp64", eta=sysm.eta)
    dev.close()
    n = npl
    rng = np.random.default_rng(7)
    for e, E in enumerate(Es):
        M = sysm.M_of_E(E)
        ref = _oracle_tri(sysm, E)
        dd = _tri_of(o_ddrgf.bndiag_of_inv_ddrgf(M, levels)[0], n)
        if eta >= 1e-2:
            bars = [2.5e-10] * 3
        else:
            pert = _tri_of(o_ddrgf.bndiag_of_inv_ddrgf(_perturbed(M, rng), levels)[0], n)
            bars = [2.5e-10 + 30.0 * max(_max_err(dd[p], ref[p]), _max_err(pert[p], dd[p])) for p in range(3)]
        for part in range(3):
            assert _max_err(f64[part][e], dd[part]) < bars[part]
            assert _max_err(mix[part][e], dd[part]) < bars[part]
            assert _max_err(rgf[part][e], ref[part]) < 1e-11


@pytest.mark.parametrize("npl,b,nE", [(6, 64, 3), (4, 512, 2), (1, 40, 2)])
def test_device_selected_inverse_nopivot(negf, npl, b, nE):
    sysm = o_phys.physics_system(npl, b, seed=32)
    Es = np.linspace(-0.5, 0.6, nE)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    res = {p: dev.selected_inverse(Es, method="selinv", precision=p, eta=sysm.eta) for p in ("fp64", "mixed")}
    dev.close()
    for e, E in enumerate(Es):
        M = sysm.M_of_E(E)
        A = {k: v for k, v in M.M.items()}
        Z = o_si.block_inverse(o_si.block_factorization(A, npl, nopivot=True), npl)
        D = np.linalg.inv(bm_convert_dense(M))
        blk = lambda i, j: D[i * b:(i + 1) * b, j * b:(j + 1) * b]  # noqa: E731
        for p, bar in (("fp64", 1e-12), ("mixed", 1e-10)):
            d, u, l = res[p]
            for i in range(npl):
                assert rel_fro(d[e][i], Z[(i, i)]) < bar
                assert rel_fro(d[e][i], blk(i, i)) < bar
            for i in range(npl - 1):
                assert rel_fro(u[e][i], Z[(i, i + 1)]) < bar and rel_fro(u[e][i], blk(i, i + 1)) < bar
                assert rel_fro(l[e][i], Z[(i + 1, i)]) < bar and rel_fro(l[e][i], blk(i + 1, i)) < bar


RIND = [1, 1, 1, 2, 3, 3, 3, 4, 5]
CIND = [1, 3, 5, 2, 3, 4, 5, 4, 5]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 1e-11)])
def test_selected_inverse_batched_reference_semantics(negf, precision, tol):
    """negf_selected_inverse_batched on the reference test's pattern
    (test_selected_inverse.jl:6-55, with fill-in) for three systems at once,
    be_getrf! semantics."""
    import ctypes
    from libnegf_b200._lib import check, ptr_array, NEGF_PREC_FP64, NEGF_PREC_MIXED
    bs, npl = 48, 5
    systems = [set_sparse_block([bs] * npl, RIND, CIND, True, seed=70 + s) for s in range(3)]
    # the fill-in pattern of the factorisation (selected_inverse.jl:41-46)
    pattern = set(systems[0].keys())
    for i in range(npl):
        for k in range(i + 1, npl):
            if (i, k) in pattern:
                for l in range(k + 1, npl):
                    if (i, l) in pattern and (k, l) not in pattern:
                        pattern |= {(k, l), (l, k)}
    dev = []
    tab = []
    for A in systems:
        blocks = {k: negf.to_device(A[k] if k in A else np.zeros((bs, bs), dtype=complex)) for k in pattern}
        dev.append(blocks)
        for i in range(npl):
            for j in range(npl):
                tab.append(blocks[(i, j)].data_ptr() if (i, j) in blocks else None)
    fill = (ctypes.c_uint8 * (npl * npl))()
    prec = NEGF_PREC_FP64 if precision == "fp64" else NEGF_PREC_MIXED
    check(negf.load().negf_selected_inverse_batched(3, npl, bs, ptr_array(tab), fill, 3, 1, prec, None))
    for A, blocks in zip(systems, dev):
        Z_ref = o_si.block_inverse(o_si.block_factorization(A, npl), npl)
        invT = np.linalg.inv(full_of_blocks(A, [bs] * npl))
        for (i, j) in Z_ref:
            z = negf.to_host(blocks[(i, j)])
            assert np.abs(z - Z_ref[(i, j)]).max() < tol
            assert np.abs(z - invT[i * bs:(i + 1) * bs, j * bs:(j + 1) * bs]).max() < tol
