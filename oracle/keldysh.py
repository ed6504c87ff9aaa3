"""Oracle restatement of the recursive Keldysh (RKD) sweep.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Computes the block tridiagonal of G^n = M^{-1} S M^{-H} for S Hermitian and
stored as diagonal + upper blocks.  Follows ``keldyshndiag_v3!``
(src/keldyshndiag.jl:166-188) and its four passes: the RGF upward pass
(:191-219), the RKD upward pass (:221-235), the central pass (:237-302) and the
RKD downward pass (:304-317).  ``buffTx`` off-diagonals are the RGF multipliers
R_i = buffM1[i,i+1] and L_{i+1} = buffM1[i+1,i].
"""

import numpy as np

from .backend_cpu import be_mldivide, be_gemm, be_ctranspose
from .blockmatrix import BlockMatrix
from .rgf import rgf_upward


def keldyshndiag(M, S, upward=None):
    """Returns the Hermitian BlockMatrix ``buffS`` (diag + upper blocks).
    ``upward`` reuses a precomputed (lu, R, L) of the RGF upward pass."""
    npl = M.npl
    lu, R, L = upward if upward is not None else rgf_upward(M)   # keldyshndiag.jl:169
    s = {k: v.copy() for k, v in S.M.items()}                    # :178  bm_copy!(buffS, S)

    # upward RKD pass (:221-235)
    for ix in range(npl - 2, -1, -1):
        s[(ix, ix)] = be_gemm("N", "C", -1.0, R[ix], s[(ix, ix + 1)], 1.0, s[(ix, ix)])          # :231
        s[(ix, ix + 1)] = be_gemm("N", "N", -1.0, R[ix], s[(ix + 1, ix + 1)], 1.0, s[(ix, ix + 1)])  # :232
        s[(ix, ix)] = be_gemm("N", "C", -1.0, s[(ix, ix + 1)], R[ix], 1.0, s[(ix, ix)])          # :233

    # central pass (:237-302)
    m2 = {}
    xb = {}
    if npl > 1:
        # the reference rescales block (1,2) unconditionally and so needs npl >= 2;
        # with one layer only the diagonal rescale below applies
        m2[(0, 1)] = be_mldivide("N", s[(0, 1)], lu[0])          # :257
        m2[(1, 0)] = be_ctranspose(m2[(0, 1)])                   # :258
        xb[(1, 0)] = be_mldivide("N", m2[(1, 0)], lu[1])         # :259
        s[(0, 1)] = be_ctranspose(xb[(1, 0)])                    # :260
    xb[(0, 0)] = np.eye(M.blockSizes[0], dtype=np.complex128)    # :263-268
    for ix in range(1, npl - 1):                                 # :270
        m2[(ix - 1, ix)] = be_gemm("N", "N", 1.0, xb[(ix - 1, ix - 1)], R[ix - 1], 0.0, None)    # :273
        xb[(ix - 1, ix)] = be_mldivide("N", m2[(ix - 1, ix)], lu[ix - 1])                       # :274
        xb[(ix, ix)] = be_gemm("N", "N", 1.0, M.M[(ix, ix - 1)], xb[(ix - 1, ix)], 0.0, None)   # :275
        xb[(ix, ix)] = xb[(ix, ix)] + np.eye(M.blockSizes[ix])                                   # :280-283
        m2[(ix, ix)] = be_mldivide("N", xb[(ix, ix)], lu[ix])                                   # :285
        m2[(ix, ix + 1)] = be_gemm("N", "N", 1.0, m2[(ix, ix)], s[(ix, ix + 1)], 0.0, None)    # :286
        m2[(ix + 1, ix)] = be_ctranspose(m2[(ix, ix + 1)])                                      # :289
        xb[(ix + 1, ix)] = be_mldivide("N", m2[(ix + 1, ix)], lu[ix + 1])                       # :290
        s[(ix, ix + 1)] = be_ctranspose(xb[(ix + 1, ix)])                                       # :291
    for ix in range(npl):                                        # :296-301
        m2[(ix, ix)] = be_mldivide("N", s[(ix, ix)], lu[ix])
        xb[(ix, ix)] = be_ctranspose(m2[(ix, ix)])
        m2[(ix, ix)] = be_mldivide("N", xb[(ix, ix)], lu[ix])
        s[(ix, ix)] = be_ctranspose(m2[(ix, ix)])

    # downward RKD pass (:304-317)
    for ix in range(npl - 1):
        s[(ix + 1, ix + 1)] = be_gemm("C", "C", -1.0, s[(ix, ix + 1)], L[ix + 1], 1.0, s[(ix + 1, ix + 1)])  # :314
        s[(ix, ix + 1)] = be_gemm("N", "C", -1.0, s[(ix, ix)], L[ix + 1], 1.0, s[(ix, ix + 1)])              # :315
        s[(ix + 1, ix + 1)] = be_gemm("N", "N", -1.0, L[ix + 1], s[(ix, ix + 1)], 1.0, s[(ix + 1, ix + 1)])  # :316

    out = BlockMatrix(S.blockSizes, S.ndiag, True)
    out.M = {k: s[k] for k in S.M.keys()}
    return out
