"""The reference's own C caller, compiled unchanged, against libnegf_b200.so.

LibNEGF.jl ships src/c_interface/libnegf_c_example.c: it builds a random
block-tridiagonal CSC matrix (160 blocks of 64), calls run_bndiag_wrapper
(libnegf_c_interface.h:22-38) and free()s the three returned arrays
(libnegf_c_example.c:99-128).  oracle/build_ref.py compiles that file as it is,
with its own header, links it to this library and adds a link-time probe
(oracle/c_example_wrap.c) that dumps the CSC input and the returned CSC band.
This test runs the program on the GPU, checks what it prints and that it
exits cleanly after freeing the arrays, and checks the returned band -- the
block tridiagonal of M^{-1} -- against the oracle's sequential RGF.  The
example draws a new matrix (uniform [0, 1] entries, time-seeded) on every run,
so its conditioning varies.  The wrapper runs DDRGF (as the reference's does,
libnegf_c_interface.jl:119) with the levels of the library's cost model; the
band's residual (M G)_ii - I, which needs only band blocks of G, is held to
10x that of the oracle's DDRGF restatement with the same levels (DDRGF's
interior-domain inverses make its residual larger than sequential RGF's), and
the forward difference to the oracle's sequential RGF to 1e-6 (measured
~5e-10).
"""

import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ROOT
from oracle import ddrgf as o_ddrgf, rgf as o_rgf
from oracle.blockmatrix import BlockMatrix

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "libnegf_c_example")


def _read_csc(path):
    with open(path, "rb") as f:
        m, n, nnz = np.frombuffer(f.read(12), dtype=np.int32)
        colptr = np.frombuffer(f.read(4 * (n + 1)), dtype=np.int32)
        rowval = np.frombuffer(f.read(4 * nnz), dtype=np.int32)
        nz = np.frombuffer(f.read(16 * nnz), dtype=np.complex128)
    return sp.csc_matrix((nz, rowval, colptr), shape=(m, n))


@pytest.mark.skipif(not os.path.exists(BIN), reason="built by oracle/build_ref.py where the reference checkout exists")
def test_reference_c_example_runs_unchanged(negf, tmp_path):
    env = dict(os.environ, NEGF_C_EXAMPLE_DUMP=str(tmp_path))
    r = subprocess.run([BIN], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    nb, b = 160, 64
    assert "Returned Matrix Size: %d x %d" % (nb * b, nb * b) in r.stdout
    assert "Returned Non-zeros: %d" % ((3 * nb - 2) * b * b) in r.stdout
    assert "Memory freed successfully" in r.stdout

    A = _read_csc(os.path.join(tmp_path, "in.bin"))
    G = _read_csc(os.path.join(tmp_path, "out.bin"))
    M = BlockMatrix([b] * nb, {"in": 3, "out": 3}, False)
    for i in range(nb):
        for j in range(max(0, i - 1), min(nb, i + 2)):
            M.M[(i, j)] = A[i * b:(i + 1) * b, j * b:(j + 1) * b].toarray()
    ref = o_rgf.bndiag_of_inv_rgf_local(M)
    got = {k: G[k[0] * b:(k[0] + 1) * b, k[1] * b:(k[1] + 1) * b].toarray() for k in ref.M}
    num = den = 0.0
    for k, blk in ref.M.items():
        num += np.linalg.norm(got[k] - blk) ** 2
        den += np.linalg.norm(blk) ** 2
    assert np.sqrt(num / den) < 1e-6

    def residual(Gb):
        worst = 0.0
        for i in range(nb):
            acc, scale = -np.eye(b), 0.0
            for j in range(max(0, i - 1), min(nb, i + 2)):
                acc = acc + M.M[(i, j)] @ Gb[(j, i)]
                scale += np.linalg.norm(M.M[(i, j)]) * np.linalg.norm(Gb[(j, i)])
            worst = max(worst, np.linalg.norm(acc) / scale)
        return worst

    levels = negf.choose_levels(nb, b, 1)
    ref_dd = o_ddrgf.bndiag_of_inv_ddrgf(M, levels)[0] if levels else ref
    assert residual(got) <= 10.0 * max(residual(ref_dd.M), residual(ref.M)) + 1e-14
