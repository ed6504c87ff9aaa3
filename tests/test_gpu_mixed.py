"""Mixed precision: complex products on the INT8 tensor cores (tcgen05) with
FP64-accurate digit splitting, against FP64.

Bars: a single product within 1e-12 relative Frobenius of the FP64 product
(the splitting carries 49 bits; measured ~1e-13); a whole batched-energy
G^R / G^< / transmission solve within 1e-10 relative Frobenius per block of
the FP64 oracle (the mixed-path tolerance of the workload).
"""

import numpy as np
import pytest

from conftest import rel_fro
from oracle import physics as o_phys

pytestmark = pytest.mark.gpu


def _rand(rng, m, n, scale=1.0):
    return scale * (rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n)))


@pytest.mark.parametrize("ops", ["NN", "NC", "CN", "CC", "TN", "NT"])
@pytest.mark.parametrize("shape", [(128, 64, 32), (256, 256, 256), (37, 45, 29), (130, 70, 257), (1, 1, 1),
                                   (200, 300, 1024), (70, 90, 512), (33, 65, 130)])
def test_mixed_gemm_vs_fp64(negf, ops, shape):
    rng = np.random.default_rng(abs(hash((ops, shape))) % 2 ** 32)
    m, n, k = shape
    tA, tB = ops
    A = _rand(rng, *((m, k) if tA == "N" else (k, m)))
    B = _rand(rng, *((k, n) if tB == "N" else (n, k)), scale=1e-3)
    C = _rand(rng, m, n)
    op = {"N": lambda x: x, "T": lambda x: x.T, "C": lambda x: x.conj().T}
    alpha, beta = -1.0, 1.0
    AB = op[tA](A) @ op[tB](B)
    ref = alpha * AB + beta * C
    dA, dB, dC = negf.to_device(A), negf.to_device(B), negf.to_device(C)
    negf.be_gemm_batched_(tA, tB, [(alpha, dA, dB, beta, dC)], precision="mixed")
    err = np.linalg.norm(negf.to_host(dC) - ref) / np.linalg.norm(AB)
    assert err < 1e-12


def test_mixed_gemm_ragged_batch_and_rows_of_zeros(negf):
    rng = np.random.default_rng(3)
    items, refs = [], []
    for (m, n, k) in [(60, 68, 61), (64, 64, 64), (3, 100, 7), (200, 5, 90)]:
        A, B, C = _rand(rng, m, k), _rand(rng, k, n), _rand(rng, m, n)
        A[0, :] = 0.0  # a zero row (scale exponent 0, all digits zero)
        refs.append((A @ B, 0.5j * (A @ B) + C))
        items.append((0.5j, negf.to_device(A), negf.to_device(B), 1.0, negf.to_device(C)))
    negf.be_gemm_batched_("N", "N", items, precision="mixed")
    for it, (ab, ref) in zip(items, refs):
        assert np.linalg.norm(negf.to_host(it[4]) - ref) / np.linalg.norm(ab) < 1e-12


@pytest.mark.parametrize("npl,b,nE", [(6, 64, 4), (4, 200, 3), (8, 48, 5)])
def test_mixed_solve_vs_oracle(negf, npl, b, nE):
    sysm = o_phys.physics_system(npl, b, seed=21)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    Es = np.linspace(-0.85, 0.7, nE)
    gr, gl, t = dev.solve(Es, eta=sysm.eta, precision="mixed")
    for e, E in enumerate(Es):
        r = o_phys.solve_energy(sysm, E)
        for i in range(npl):
            assert rel_fro(gr[e][i], r["GR"].M[(i, i)]) < 1e-10
            assert rel_fro(gl[e][i], 1j * r["Gn"].M[(i, i)]) < 1e-10
        assert abs(t[e] - r["T"]) <= 1e-10 * max(1.0, abs(r["T"]))


@pytest.mark.parametrize("b", [256, 512])
def test_mixed_solve_int8_inversion_updates(negf, b):
    """gj_update=2: the Gauss-Jordan rank-nb updates (panel widths 32 and 16
    here) as 34-pair INT8 digit products; the same bar against the oracle as
    the default FP64 updates, and both forms within 1e-10 of each other."""
    sysm = o_phys.physics_system(3, b, seed=5)
    dev = negf.Device(sysm.Hd, sysm.Hu, sysm.sigL, sysm.sigR)
    Es = np.array([-0.6, 0.25])
    gr2, gl2, t2 = dev.solve(Es, eta=sysm.eta, precision="mixed", gj_update=2)
    gr1, gl1, t1 = dev.solve(Es, eta=sysm.eta, precision="mixed", gj_update=1)
    for e, E in enumerate(Es):
        r = o_phys.solve_energy(sysm, E)
        for i in range(3):
            assert rel_fro(gr2[e][i], r["GR"].M[(i, i)]) < 1e-10
            assert rel_fro(gl2[e][i], 1j * r["Gn"].M[(i, i)]) < 1e-10
            assert rel_fro(gr2[e][i], gr1[e][i]) < 1e-10
        assert abs(t2[e] - r["T"]) <= 1e-10 * max(1.0, abs(r["T"]))
    dev.close()
