"""Oracle restatement of the block n-diagonal (bandwidth w) RGF.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows ``bndiag_of_inv_general_rgf!`` (src/matinvertndiag_general_rgf.jl:31-146).
The reference overwrites ``Min`` with the Schur-updated blocks (:86); the oracle
works on a copy so the caller's matrix is unchanged (the in-place variant is
``overwrite=True``).
"""

import numpy as np

from .backend_cpu import be_lu, be_mldivide, be_gemm, be_ctranspose, be_identity
from .blockmatrix import BlockMatrix, bm_copy


def bndiag_of_inv_general_rgf(Min, overwrite=False, build_full_inv=False):
    M = Min if overwrite else bm_copy(Min)
    npl = M.npl
    w = (M.ndiag["in"] - 1) // 2
    A = M.M
    lu = [None] * npl
    B = {}   # buffM1 off-diagonal blocks: right multipliers (t, ix+1), left multipliers (ix+1, t)
    lu[npl - 1] = be_lu(A[(npl - 1, npl - 1)])                               # :49
    for ix in range(npl - 2, -1, -1):                                         # :52
        kmax = min(w, ix + 1)
        for k in range(1, kmax + 1):                                          # :56
            t = ix - k + 1
            y = be_mldivide("C", be_ctranspose(A[(t, ix + 1)]), lu[ix + 1])   # :61-62
            B[(t, ix + 1)] = be_ctranspose(y)                                 # :63
            B[(ix + 1, t)] = be_mldivide("N", A[(ix + 1, t)], lu[ix + 1])     # :66
        for i in range(1, kmax + 1):                                          # :70
            for j in range(1, kmax + 1):
                r, c = ix - i + 1, ix - j + 1
                X = be_gemm("N", "N", -1.0, A[(r, ix + 1)], B[(ix + 1, c)], 1.0, A[(r, c)])  # :75-78
                if r == c == ix:
                    lu[ix] = be_lu(X)                                         # :82
                else:
                    A[(r, c)] = X                                             # :84
    out = BlockMatrix(M.blockSizes, {"in": M.ndiag["in"], "out": M.ndiag["in"]}, False)
    G = out.M
    G[(0, 0)] = be_mldivide("N", be_identity(M.blockSizes[0]), lu[0])        # :95
    for ix in range(1, npl):                                                  # :98
        kmax = min(w, ix)
        for k in range(1, kmax + 1):
            tp = ix - k
            up = np.zeros((M.blockSizes[tp], M.blockSizes[ix]), dtype=np.complex128)   # :105
            lo = np.zeros((M.blockSizes[ix], M.blockSizes[tp]), dtype=np.complex128)   # :106
            for k2 in range(1, kmax + 1):                                     # :109
                m = ix - k2
                up = be_gemm("N", "N", -1.0, G[(tp, m)], B[(m, ix)], 1.0, up)          # :113
                lo = be_gemm("N", "N", -1.0, B[(ix, m)], G[(m, tp)], 1.0, lo)          # :116
            G[(tp, ix)] = up
            G[(ix, tp)] = lo
        d = be_mldivide("N", be_identity(M.blockSizes[ix]), lu[ix])          # :121
        for k2 in range(1, kmax + 1):                                         # :122
            m = ix - k2
            d = be_gemm("N", "N", -1.0, B[(ix, m)], G[(m, ix)], 1.0, d)       # :124
        G[(ix, ix)] = d
    if build_full_inv and npl > 2:                                            # :129-143
        out.ndiag = {"in": M.ndiag["in"], "out": 2 * npl - 1}
        for ix in range(npl):
            for jx in range(ix + w + 1, npl):
                up = np.zeros((M.blockSizes[ix], M.blockSizes[jx]), dtype=np.complex128)
                lo = np.zeros((M.blockSizes[jx], M.blockSizes[ix]), dtype=np.complex128)
                for m in range(jx - w, jx):
                    up = be_gemm("N", "N", -1.0, G[(ix, m)], B[(m, jx)], 1.0, up)
                    lo = be_gemm("N", "N", -1.0, B[(jx, m)], G[(m, ix)], 1.0, lo)
                G[(ix, jx)] = up
                G[(jx, ix)] = lo
    return out
