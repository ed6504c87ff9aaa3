"""Batched selected inverse and DDRGF over energies, FP64 and mixed precision.

The configuration these cover: the selected inverse (tridiagonal blocks of
G^R(E) = M(E)^{-1}) of one device for many energies, by domain-decomposed RGF
(bndiag_of_inv_ddrgf!, src/matinvertndiag_ddrgf_core.jl:719-758, four
partitions) and by the block selected inverse (Block_factorization! +
Block_inverse!, src/selected_inverse.jl:9-206), every recursion step one
launch over all energies, with the block products in FP64 or on the INT8
tensor cores (mixed).

Bars: DDRGF (both precisions) against the oracle's DDRGF restatement with the
same levels, within 2.5e-10 (the reference's DDRGF tolerance,
test_matinvertndiag_ddrgf.jl:245-293) plus 10x that restatement's own distance
from sequential RGF: on the NEGF generator the interior domains are closed
systems (eta = 1e-6) whose inverses are ill-conditioned, so DDRGF itself -- the
reference's algorithm, restated on the CPU -- departs from RGF by up to ~1e-8
here, and two FP64 executions of it differ by that order; the selected inverse on the
NEGF generator (lu(NoPivot()) diagonal factorisations) against the oracle's
restatement with the same factorisation and the dense inverse at 1e-12 (FP64)
/ 1e-10 (mixed); the batched reference-API entry point against the oracle's
restatement of the reference (be_getrf! with discarded pivots) on the
reference test's diagonally dominant generator at 1e-13 absolute.
"""

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


@pytest.mark.parametrize("npl,b,nE,levels", [(16, 512, 4, [3]), (19, 64, 5, [4]), (40, 32, 3, [3, 3])])
def test_device_ddrgf_fp64_and_mixed(negf, npl, b, nE, levels):
    """DDRGF of the NEGF generator over energies; (16, 512, [3]) is the
    benchmark's b = 512 with four partitions (separators at layers 0, 4, 8, 12)."""
    sysm = o_phys.physics_system(npl, b, seed=31)
    Es = np.linspace(-0.7, 0.8, nE)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    f64 = dev.selected_inverse(Es, method="ddrgf", precision="fp64", eta=sysm.eta, levels=levels)
    mix = dev.selected_inverse(Es, method="ddrgf", precision="mixed", eta=sysm.eta, levels=levels)
    rgf = dev.selected_inverse(Es, method="rgf", precision="fp64", eta=sysm.eta)
    dev.close()
    n = npl
    for e, E in enumerate(Es):
        ref = _oracle_tri(sysm, E)
        D = o_ddrgf.bndiag_of_inv_ddrgf(sysm.M_of_E(E), levels)[0]
        dd = ([D.M[(i, i)] for i in range(n)], [D.M[(i, i + 1)] for i in range(n - 1)],
              [D.M[(i + 1, i)] for i in range(n - 1)])
        for part in range(3):
            bar = 2.5e-10 + 10.0 * _max_err(dd[part], ref[part])
            assert _max_err(f64[part][e], dd[part]) < bar
            assert _max_err(mix[part][e], dd[part]) < bar
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
